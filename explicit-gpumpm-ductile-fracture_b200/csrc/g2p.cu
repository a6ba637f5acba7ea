// G2P: grid-to-particle transfer (G2P_APIC, G2PKernal.cu:204-441) fused with
// the constitutive update that the reference runs at the start of the next
// substep (applyVonMises, ExplicitTimeIntegrator.cu:132-370) and with the
// phase-field gradient gather (AxG2P_APIC, G2PKernal.cu:1006-1123).
//
// Each CTA takes an equal share of the sorted slots and walks it in units of
// up to 256 slots that run across page boundaries.  For every page it stages
// the 6x6x6 window of v, dc and c_new in shared memory; one thread per
// particle then gathers its 3x3x3 stencil, updates c
// (irreversibly), x, F = (I + dt grad v) F, the APIC matrix B, runs the SVD +
// Hencky return map + damage driving force, and writes the particle in the
// new sorted order, with the cell key and page flag of its new position for
// the next substep's binning (cal_cellId, Particle_kernal.cu:158-165, done
// where the position is written instead of in a pass that reads it back).
// Reading the previous order through perm and writing the
// new order is the reorder the reference does with gathers and D2D copies
// (Particle_kernal.cu:544-573, TimeIntegrator.cu:459-461).
#include <algorithm>
#include <cstdint>

#include "async_copy.cuh"
#include "constitutive.cuh"
#include "kernels.h"
#include "launch.cuh"

namespace gmpm {

// Work unit: up to kG2PUnit consecutive sorted slots of the CTA's share,
// spanning at most kUnitPages pages, so that no thread slot idles at a page
// end (a page of 385 particles no longer costs a unit of 256 and one of 129).
// A CTA walks its units with a three-deep software pipeline of asynchronous
// copies:
//   unit k+2: perm, sorted keys, and its pages' adjacency rows and keys  (meta)
//   unit k+1: the particles' inputs through perm (x, c, m, id one value per
//             copy; F, alpha and psi_max as three four-wide words, one
//             16-byte copy each in FP32) and the 6x6x6
//             node window of each page not staged yet                    (data)
//   unit k  : computed from shared memory
// so global latency is hidden behind the previous unit's arithmetic.  Pages
// are numbered in the order the CTA meets them; a page's window sits in ring
// slot seq mod kWinRing and its adjacency row and key in slot seq mod
// kPageRing (units k .. k+2 span at most 9 pages, units k and k+1 at most 6).
constexpr int kG2PUnit = 256;
constexpr int kG2PMinBlocks = 2;  // resident CTAs per SM (FP32), bounded by registers
constexpr int kPlanesR = 5;   // x0..2, c, m (F, alpha and psi travel as three words)
constexpr int kUnitPages = 3;
constexpr int kWinRing = 8;
constexpr int kPageRing = 16;

// Unit descriptor fields in shared memory.
enum : int { UD_S0 = 0, UD_N = 1, UD_SEQ = 2, UD_NP = 3, UD_C1 = 4, UD_C2 = 5, UD_P0 = 6, UD_WORDS = 8 };

template <typename R>
struct G2PShared {
    R win4[kWinRing][kWindowNodes][4];  // (v0, v1, v2, dc) per window node
    R wincn[kWinRing][kWindowNodes];    // c_new per window node
    R p[2][kPlanesR][kG2PUnit];          // staged particle inputs; 2 unit buffers
    Word4<R> pw[2][3][kG2PUnit];         // staged F / alpha / psi words; 2 unit buffers
    uint32_t id[2][kG2PUnit];
    int32_t o[3][kG2PUnit];              // previous slot per unit slot; 3 meta buffers
    uint32_t key[3][kG2PUnit];
    int32_t adj[kPageRing][8];
    uint32_t bkey[kPageRing];
    int32_t unit[3][UD_WORDS];
    // per window value w = ch * 216 + node: source offset in its grid page
    // (bits 0-8), neighbour slot (9-11), destination offset (12-21), c_new flag (22)
    uint32_t wtab[kGridChannels * kWindowNodes];
    // the cell-key parameters, read where each particle's key is formed (not
    // held in registers across the loop)
    double key_inv_dx;
    int key_res[3];
};

enum : int { P_X = 0, P_C = 3, P_M = 4 };

// One particle word: one 16-byte copy in FP32, two in FP64.
template <typename R>
__device__ __forceinline__ void cp_async_word(Word4<R>* dst, const Word4<R>* src) {
    static_assert(sizeof(Word4<R>) % 16 == 0, "whole 16-byte copies");
#pragma unroll
    for (int h = 0; h < (int)(sizeof(Word4<R>) / 16); ++h)
        cp_async<16>(reinterpret_cast<char*>(dst) + 16 * h, reinterpret_cast<const char*>(src) + 16 * h);
}

// quadratic B-spline weights and gradients on nodes base+0..2 along one axis,
// xp relative to the base node (G2PKernal.cu:257-288)
template <typename R>
__device__ __forceinline__ void bspline1d_g(R xp, R inv_dx, R* w, R* g) {
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

// Gather of v, dc, grad v, B and grad c over the particle's 3x3x3 stencil
// (G2PKernal.cu:286-357, AxG2P_APIC :1085-1112) from the page's staged window
// (li, lj, lk: the base node's offset in the window).  The weights are tensor
// products w = X_i Y_j Z_k, and the APIC offset x_i - x_p splits per axis, so
// the sums are taken one axis at a time: over k for each (i, j) column, then
// over j, then over i.
template <typename R>
__device__ __forceinline__ void gather_stencil(const R (*__restrict__ win4)[4], const R* __restrict__ wincn, int li,
                                               int lj, int lk, const R xp[3], R dx, const R wx[3], const R gx[3],
                                               const R wy[3], const R gy[3], const R wz[3], const R gz[3], R vp[3],
                                               R& dcp, R gv[9], R Bn[9], R gc[3]) {
    vp[0] = vp[1] = vp[2] = dcp = R(0);
    gc[0] = gc[1] = gc[2] = R(0);
#pragma unroll
    for (int q = 0; q < 9; ++q) gv[q] = Bn[q] = R(0);
    R wxd[3], wyd[3], wzd[3];  // weight x (node - particle) offset per axis
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        wxd[q] = wx[q] * (R(q) * dx - xp[0]);
        wyd[q] = wy[q] * (R(q) * dx - xp[1]);
        wzd[q] = wz[q] * (R(q) * dx - xp[2]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        // sums over j for this i: T0 (Y Z), Ty (Y' Z), Tz (Y Z'), Tdy (Y d Z), Tdz (Y Z d)
        R T0[3], Ty[3], Tz[3], Tdy[3], Tdz[3], Td = R(0), Tc0 = R(0), Tcy = R(0), Tcz = R(0);
#pragma unroll
        for (int a = 0; a < 3; ++a) T0[a] = Ty[a] = Tz[a] = Tdy[a] = Tdz[a] = R(0);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            // sums over k for column (i, j): Z0 (Z), Z1 (Z'), Z2 (Z d)
            R Z0[3], Z1[3], Z2[3], Zd = R(0), C0 = R(0), C1 = R(0);
#pragma unroll
            for (int a = 0; a < 3; ++a) Z0[a] = Z1[a] = Z2[a] = R(0);
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
                const int node = (li + i) * 36 + (lj + j) * 6 + (lk + kk);
                R nv[4];
                if (sizeof(R) == 4) {
                    *reinterpret_cast<float4*>(nv) = *reinterpret_cast<const float4*>(&win4[node][0]);
                } else {
                    *reinterpret_cast<double2*>(nv) = *reinterpret_cast<const double2*>(&win4[node][0]);
                    *reinterpret_cast<double2*>(nv + 2) = *reinterpret_cast<const double2*>(&win4[node][2]);
                }
                const R ncn = wincn[node];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    Z0[a] += wz[kk] * nv[a];
                    Z1[a] += gz[kk] * nv[a];
                    Z2[a] += wzd[kk] * nv[a];
                }
                Zd += wz[kk] * nv[3];
                C0 += wz[kk] * ncn;
                C1 += gz[kk] * ncn;
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                T0[a] += wy[j] * Z0[a];
                Ty[a] += gy[j] * Z0[a];
                Tz[a] += wy[j] * Z1[a];
                Tdy[a] += wyd[j] * Z0[a];
                Tdz[a] += wy[j] * Z2[a];
            }
            Td += wy[j] * Zd;
            Tc0 += wy[j] * C0;
            Tcy += gy[j] * C0;
            Tcz += wy[j] * C1;
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            vp[a] += wx[i] * T0[a];
            gv[a + 0] += gx[i] * T0[a];
            gv[a + 3] += wx[i] * Ty[a];
            gv[a + 6] += wx[i] * Tz[a];
            Bn[a + 0] += wxd[i] * T0[a];
            Bn[a + 3] += wx[i] * Tdy[a];
            Bn[a + 6] += wx[i] * Tdz[a];
        }
        dcp += wx[i] * Td;
        gc[0] += gx[i] * Tc0;
        gc[1] += wx[i] * Tcy;
        gc[2] += wx[i] * Tcz;
    }
}

// FP32: the same sums, two channels per packed instruction (fma.rn.f32x2).
// Every value is the same fused multiply-add, in the same order, as in the
// scalar form; the window's (v0, v1) and (v2, dc) halves of each 16-byte node
// word are the packed operands, the weights are broadcast to both halves.
template <>
__device__ __forceinline__ void gather_stencil<float>(const float (*__restrict__ win4)[4],
                                                      const float* __restrict__ wincn, int li, int lj, int lk,
                                                      const float xp[3], float dx, const float wx[3],
                                                      const float gx[3], const float wy[3], const float gy[3],
                                                      const float wz[3], const float gz[3], float vp[3], float& dcp,
                                                      float gv[9], float Bn[9], float gc[3]) {
    float wxd[3], wyd[3], wzd[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        wxd[q] = wx[q] * (float(q) * dx - xp[0]);
        wyd[q] = wy[q] * (float(q) * dx - xp[1]);
        wzd[q] = wz[q] * (float(q) * dx - xp[2]);
    }
    const float2 zero = make_float2(0.f, 0.f);
    // accumulators: pairs of channels (x, y components), then the z component alone,
    // or (z component, damage increment) where both take the same weight
    float2 VP01 = zero, VP2D = zero, GV01 = zero, GV34 = zero, GV67 = zero, B01 = zero, B34 = zero, B67 = zero;
    float gv2 = 0.f, gv5 = 0.f, gv8 = 0.f, b2 = 0.f, b5 = 0.f, b8 = 0.f, gc0 = 0.f, gc1 = 0.f, gc2 = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float2 T001 = zero, T02D = zero, Ty01 = zero, Tz01 = zero, Tdy01 = zero, Tdz01 = zero;
        float Ty2 = 0.f, Tz2 = 0.f, Tdy2 = 0.f, Tdz2 = 0.f, Tc0 = 0.f, Tcy = 0.f, Tcz = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float2 Z001 = zero, Z02D = zero, Z101 = zero, Z201 = zero;
            float Z12 = 0.f, Z22 = 0.f, C0 = 0.f, C1 = 0.f;
#pragma unroll
            for (int kk = 0; kk < 3; ++kk) {
                const int node = (li + i) * 36 + (lj + j) * 6 + (lk + kk);
                const float4 nv = *reinterpret_cast<const float4*>(&win4[node][0]);
                const float2 n01 = make_float2(nv.x, nv.y), n2d = make_float2(nv.z, nv.w);
                const float ncn = wincn[node];
                const float2 W = make_float2(wz[kk], wz[kk]), G = make_float2(gz[kk], gz[kk]);
                const float2 WD = make_float2(wzd[kk], wzd[kk]);
                Z001 = __ffma2_rn(W, n01, Z001);
                Z02D = __ffma2_rn(W, n2d, Z02D);
                Z101 = __ffma2_rn(G, n01, Z101);
                Z12 = __fmaf_rn(gz[kk], nv.z, Z12);
                Z201 = __ffma2_rn(WD, n01, Z201);
                Z22 = __fmaf_rn(wzd[kk], nv.z, Z22);
                C0 = __fmaf_rn(wz[kk], ncn, C0);
                C1 = __fmaf_rn(gz[kk], ncn, C1);
            }
            const float2 WY = make_float2(wy[j], wy[j]), GY = make_float2(gy[j], gy[j]);
            const float2 WYD = make_float2(wyd[j], wyd[j]);
            T001 = __ffma2_rn(WY, Z001, T001);
            T02D = __ffma2_rn(WY, Z02D, T02D);
            Ty01 = __ffma2_rn(GY, Z001, Ty01);
            Ty2 = __fmaf_rn(gy[j], Z02D.x, Ty2);
            Tz01 = __ffma2_rn(WY, Z101, Tz01);
            Tz2 = __fmaf_rn(wy[j], Z12, Tz2);
            Tdy01 = __ffma2_rn(WYD, Z001, Tdy01);
            Tdy2 = __fmaf_rn(wyd[j], Z02D.x, Tdy2);
            Tdz01 = __ffma2_rn(WY, Z201, Tdz01);
            Tdz2 = __fmaf_rn(wy[j], Z22, Tdz2);
            Tc0 = __fmaf_rn(wy[j], C0, Tc0);
            Tcy = __fmaf_rn(gy[j], C0, Tcy);
            Tcz = __fmaf_rn(wy[j], C1, Tcz);
        }
        const float2 WX = make_float2(wx[i], wx[i]), GX = make_float2(gx[i], gx[i]);
        const float2 WXD = make_float2(wxd[i], wxd[i]);
        VP01 = __ffma2_rn(WX, T001, VP01);
        VP2D = __ffma2_rn(WX, T02D, VP2D);
        GV01 = __ffma2_rn(GX, T001, GV01);
        gv2 = __fmaf_rn(gx[i], T02D.x, gv2);
        GV34 = __ffma2_rn(WX, Ty01, GV34);
        gv5 = __fmaf_rn(wx[i], Ty2, gv5);
        GV67 = __ffma2_rn(WX, Tz01, GV67);
        gv8 = __fmaf_rn(wx[i], Tz2, gv8);
        B01 = __ffma2_rn(WXD, T001, B01);
        b2 = __fmaf_rn(wxd[i], T02D.x, b2);
        B34 = __ffma2_rn(WX, Tdy01, B34);
        b5 = __fmaf_rn(wx[i], Tdy2, b5);
        B67 = __ffma2_rn(WX, Tdz01, B67);
        b8 = __fmaf_rn(wx[i], Tdz2, b8);
        gc0 = __fmaf_rn(gx[i], Tc0, gc0);
        gc1 = __fmaf_rn(wx[i], Tcy, gc1);
        gc2 = __fmaf_rn(wx[i], Tcz, gc2);
    }
    vp[0] = VP01.x; vp[1] = VP01.y; vp[2] = VP2D.x; dcp = VP2D.y;
    gv[0] = GV01.x; gv[1] = GV01.y; gv[2] = gv2;
    gv[3] = GV34.x; gv[4] = GV34.y; gv[5] = gv5;
    gv[6] = GV67.x; gv[7] = GV67.y; gv[8] = gv8;
    Bn[0] = B01.x; Bn[1] = B01.y; Bn[2] = b2;
    Bn[3] = B34.x; Bn[4] = B34.y; Bn[5] = b5;
    Bn[6] = B67.x; Bn[7] = B67.y; Bn[8] = b8;
    gc[0] = gc0; gc[1] = gc1; gc[2] = gc2;
}

// Unit sequence of one CTA: slots [b T / C, (b + 1) T / C) of the T sorted
// slots, b the CTA's index and C the CTA count of its scene's share of the
// launch, in units of up to kG2PUnit slots and kUnitPages pages.
// Every thread runs the same iterator in step (it shuffles), so it is called
// by all threads of the CTA at the same points.  Page starts cs(q) =
// cell_start[64 q] are held 32 pages at a time in lane registers, the next
// 32 prefetched.
struct UnitIter {
    int64_t s, se;    // next unit start, end of the CTA's share
    int p, seq;       // page containing s and its sequence number
    int nb, total;
    int P0;           // first page of the lane-held block
    int cur, nxt;     // cs(P0 + lane), cs(P0 + 32 + lane)
    __device__ int load_cs(const BinDev& bin, int q) const {
        q = min(q, nb);
        return bin.cell_start[(int64_t)q * 64];
    }
    __device__ void init(const BinDev& bin, int nb_, VB vb) {
        nb = nb_;
        total = nb > 0 ? bin.cell_start[(int64_t)nb * 64] : 0;
        s = (int64_t)vb.b * total / vb.g;
        se = (int64_t)(vb.b + 1) * total / vb.g;
        p = 0;
        if (s < se) p = bin.page_rank[bin.keys_sorted[s] >> 6];
        seq = 0;
        P0 = p;
        const int lane = threadIdx.x & 31;
        cur = load_cs(bin, P0 + lane);
        nxt = load_cs(bin, P0 + 32 + lane);
    }
    // cs(q) for P0 <= q < P0 + 64
    __device__ int cs(int q) const {
        const int r = q - P0;
        const int lo = __shfl_sync(0xffffffffu, cur, r & 31);
        const int hi = __shfl_sync(0xffffffffu, nxt, r & 31);
        return r < 32 ? lo : hi;
    }
    // Next unit; n = 0 when the CTA is done.
    __device__ void step(const BinDev& bin, int& s0, int& n, int& seq0, int& np, int& c1, int& c2, int& p0) {
        // keep p in the first block, so that p .. p + kUnitPages lie in the two
        while (p >= P0 + 32) {
            P0 += 32;
            cur = nxt;
            nxt = load_cs(bin, P0 + 32 + (int)(threadIdx.x & 31));
        }
        if (s >= se) {
            s0 = n = seq0 = np = c1 = c2 = p0 = 0;
            return;
        }
        const int a1 = cs(p + 1), a2 = cs(p + 2), a3 = cs(p + 3);
        int64_t e = min(s + kG2PUnit, se);
        if (a3 < e) e = a3;
        s0 = (int)s;
        n = (int)(e - s);
        seq0 = seq;
        p0 = p;
        np = 1 + (a1 < e) + (a2 < e);
        c1 = a1;
        c2 = a2;
        const int adv = (a1 <= e) + (a2 <= e) + (a3 <= e);
        p += adv;
        seq += adv;
        s = e;
    }
};

template <typename R>
__device__ __forceinline__ void issue_meta(G2PShared<R>& S, int m, int s0, int n, int seq0, int np, int p0,
                                           const BinDev& bin) {
    const int t = threadIdx.x;
    if (n <= 0) return;
    if (t < n) {
        cp_async_elem(&S.o[m][t], &bin.perm[s0 + t]);
        cp_async_elem(&S.key[m][t], &bin.keys_sorted[s0 + t]);
    }
    if (t < 8 * np) {
        const int j = t >> 3;
        cp_async_elem(&S.adj[(seq0 + j) % kPageRing][t & 7], &bin.adj[(int64_t)(p0 + j) * 8 + (t & 7)]);
    } else if (t < 8 * kUnitPages + np && t >= 8 * kUnitPages) {
        const int j = t - 8 * kUnitPages;
        cp_async_elem(&S.bkey[(seq0 + j) % kPageRing], &bin.block_keys[p0 + j]);
    }
}

// Particle inputs of a unit, and the windows of its pages with sequence
// numbers in [wseq0, wseq1) (the pages not staged by the previous unit).
template <typename R>
__device__ __forceinline__ void issue_data(G2PShared<R>& S, int m, int buf, int n, int wseq0, int wseq1,
                                           const PState<R>& in, const R* __restrict__ nodes) {
    const int t = threadIdx.x;
    if (t < n) {
        const int o = S.o[m][t];
#pragma unroll
        for (int a = 0; a < 3; ++a) cp_async_elem(&S.p[buf][P_X + a][t], in.x[a] + o);
#pragma unroll
        for (int k = 0; k < 3; ++k) cp_async_word(&S.pw[buf][k][t], in.fw[k] + o);
        cp_async_elem(&S.p[buf][P_C][t], in.c + o);
        cp_async_elem(&S.p[buf][P_M][t], in.m + o);
        cp_async_elem(&S.id[buf][t], in.id + o);
    }
    for (int wseq = wseq0; wseq < wseq1; ++wseq) {
        const int wbuf = wseq % kWinRing;
        const int32_t* adj = S.adj[wseq % kPageRing];
        for (int w = t; w < kGridChannels * kWindowNodes; w += kG2PUnit) {
            const uint32_t e = S.wtab[w];
            const int g = adj[(e >> 9) & 7];
            const int off = (int)((e >> 12) & 1023);
            R* dst = (e >> 22) ? &S.wincn[wbuf][off] : &S.win4[wbuf][0][0] + off;
            if (g >= 0)
                cp_async_elem(dst, nodes + (int64_t)g * kGridChannels * 64 + (e & 511));
            else
                *dst = R(0);
        }
    }
}

// kAnyModel: a material uses an energy model other than von Mises.
// kFallback: the scene redoes the SVD and return map in FP64 for ill-conditioned F
// (FP32 with the FP64 fallback).  The fallback's FP64 registers make the FP32
// kernel spill (76-136 bytes at 128 registers), so scenes without it launch
// the instantiation that leaves it out (126 registers, no spills).
template <typename R, bool kAnyModel, bool kFallback>
__device__ __forceinline__ void g2p_body(VB vb, const SceneDev<R>* __restrict__ sc,
                                         const SceneDev<double>* __restrict__ sc64, const PState<R>& in,
                                         const PState<R>& out, const PAux<R>& aux, const BinDev& bin,
                                         const R* __restrict__ nodes, Counters* cnt) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    G2PShared<R>& S = *reinterpret_cast<G2PShared<R>*>(smem_raw);
    const int t = threadIdx.x;
    const int nb = min(cnt->n_blocks, bin.nb_cap);
    const R dx = sc->dx, inv_dx = sc->inv_dx, dt = sc->dt, V0 = sc->V0;
    const bool fallback = kFallback && sc->fp64_svd_fallback && sc64 != nullptr;
    const R ratio = sc->svd_fallback_ratio;
    unsigned int flags = 0;
    double v2max = 0.0;  // max |v_p|^2 of this thread's particles (adaptive dt)

    // prologue: meta of units 0 and 1, data of unit 0
    UnitIter it;
    it.init(bin, nb, vb);
    int d0[7], d1[7];  // s0, n, seq0, np, c1, c2, p0
    it.step(bin, d0[0], d0[1], d0[2], d0[3], d0[4], d0[5], d0[6]);
    it.step(bin, d1[0], d1[1], d1[2], d1[3], d1[4], d1[5], d1[6]);
    if (t == 0) {
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            S.unit[0][q] = d0[q];
            S.unit[1][q] = d1[q];
        }
        S.key_inv_dx = sc->inv_dx_d;
        for (int a = 0; a < 3; ++a) S.key_res[a] = sc->res[a];
    }
    issue_meta(S, 0, d0[0], d0[1], d0[2], d0[3], d0[6], bin);
    cp_async_commit();
    // window copy table, once per CTA (the divisions of the node index)
    for (int w = t; w < kGridChannels * kWindowNodes; w += kG2PUnit) {
        const int ch = w / kWindowNodes;
        const int node = w - ch * kWindowNodes;
        const int a = node / 36, bb = (node / 6) % 6, cc = node % 6;
        const int d = ((a >> 2) << 2) | ((bb >> 2) << 1) | (cc >> 2);
        const uint32_t src = (uint32_t)(ch * 64 + (a & 3) * 16 + (bb & 3) * 4 + (cc & 3));
        const uint32_t dst = (uint32_t)(ch < 4 ? node * 4 + ch : node);
        S.wtab[w] = src | ((uint32_t)d << 9) | (dst << 12) | ((uint32_t)(ch == 4) << 22);
    }
    cp_async_wait_all();
    __syncthreads();
    int staged = d0[2] + d0[3];  // pages with sequence numbers below this have their window staged
    issue_data(S, 0, 0, d0[1], d0[1] > 0 ? d0[2] : 0, d0[1] > 0 ? staged : 0, in, nodes);
    issue_meta(S, 1, d1[0], d1[1], d1[2], d1[3], d1[6], bin);
    cp_async_commit();

    for (int k = 0;; ++k) {
        cp_async_wait_all();
        __syncthreads();
        const int m0 = k % 3, m1 = (k + 1) % 3, m2 = (k + 2) % 3;
        const int u0s = S.unit[m0][UD_S0], u0n = S.unit[m0][UD_N], u0seq = S.unit[m0][UD_SEQ];
        const int u0c1 = S.unit[m0][UD_C1], u0c2 = S.unit[m0][UD_C2], u0np = S.unit[m0][UD_NP];
        if (u0n <= 0) break;
        {
            // unit k+2: iterator step, descriptor and meta; unit k+1: data
            int d2[7];
            it.step(bin, d2[0], d2[1], d2[2], d2[3], d2[4], d2[5], d2[6]);
            const int u1n = S.unit[m1][UD_N], u1seq = S.unit[m1][UD_SEQ], u1np = S.unit[m1][UD_NP];
            if (t == 0) {
#pragma unroll
                for (int q = 0; q < 7; ++q) S.unit[m2][q] = d2[q];
            }
            int w0 = 0, w1 = 0;
            if (u1n > 0) {
                w0 = max(u1seq, staged);
                w1 = u1seq + u1np;
                staged = max(staged, w1);
            }
            issue_data(S, m1, (k + 1) & 1, u1n, w0, w1, in, nodes);
            issue_meta(S, m2, d2[0], d2[1], d2[2], d2[3], d2[6], bin);
            cp_async_commit();
        }
        if (t < u0n) {
            const int buf = k & 1;
            const int slot = u0s + t;
            // the particle's page within the unit
            const int pseq = u0seq + (u0np > 1 && slot >= u0c1) + (u0np > 2 && slot >= u0c2);
            int bx, by, bz;
            page_coords(S.bkey[pseq % kPageRing], bx, by, bz);
            const uint32_t cell = S.key[m0][t] & 63u;
            const int li = (int)(cell >> 4), lj = (int)((cell >> 2) & 3), lk = (int)(cell & 3);
            const R x[3] = {S.p[buf][P_X][t], S.p[buf][P_X + 1][t], S.p[buf][P_X + 2][t]};
            const R xp[3] = {x[0] - R(4 * bx + li) * dx, x[1] - R(4 * by + lj) * dx, x[2] - R(4 * bz + lk) * dx};
            R wx[3], gx[3], wy[3], gy[3], wz[3], gz[3];
            bspline1d_g(xp[0], inv_dx, wx, gx);
            bspline1d_g(xp[1], inv_dx, wy, gy);
            bspline1d_g(xp[2], inv_dx, wz, gz);
            // Gather of v, dc, grad v, B and grad c over the 3x3x3 stencil
            // (G2PKernal.cu:286-357, AxG2P_APIC :1085-1112).  The weights are
            // tensor products w = X_i Y_j Z_k, and the APIC offset x_i - x_p
            // splits per axis, so the sums are taken one axis at a time: over
            // k for each (i, j) column, then over j, then over i.
            R vp[3], dcp, gv[9], Bn[9], gc[3];
            gather_stencil(S.win4[pseq % kWinRing], S.wincn[pseq % kWinRing], li, lj, lk, xp, dx, wx, gx, wy, gy,
                           wz, gz, vp, dcp, gv, Bn, gc);
            // damage: irreversible (G2PKernal.cu:359-366)
            const R c_old = S.p[buf][P_C][t];
            const R c_new = fmax(fmin(c_old, c_old + dcp), R(0));
            // Write the transfer results first so they are dead during the SVD.
            bool finite = true;
            R xn[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                xn[a] = x[a] + vp[a] * dt;
                out.x[a][slot] = xn[a];
                aux.v[a][slot] = vp[a];
                finite = finite && isfinite(xn[a]);
            }
            {
                // the new position's cell key and page, which the next
                // substep's binning reads instead of running its key pass
                bool bad = false;
                const uint32_t key = cell_key(xn, S.key_inv_dx, S.key_res, bad);
                bin.keys[slot] = key;
                bin.page_flag[key >> 6] = 1;
                if (bad) flags |= GMPM_FLAG_OUT_OF_DOMAIN;
            }
#pragma unroll
            for (int q = 0; q < 9; ++q) aux.B[q][slot] = Bn[q];
            if (sc->adaptive_dt) v2max = fmax(v2max, (double)(vp[0] * vp[0] + vp[1] * vp[1] + vp[2] * vp[2]));
            out.c[slot] = c_new;
            out.m[slot] = S.p[buf][P_M][t];
            const uint32_t idw = S.id[buf][t];
            out.id[slot] = idw;
            // F <- (I + dt grad v) F  (G2PKernal.cu:372-404)
            const Word4<R> w0 = S.pw[buf][0][t], w1 = S.pw[buf][1][t], w2 = S.pw[buf][2][t];
            const R Fi[9] = {w0.v[0], w0.v[1], w0.v[2], w0.v[3], w1.v[0], w1.v[1], w1.v[2], w1.v[3], w2.v[0]};
            R Fo[9];
            {
                R A[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) A[q] = gv[q] * dt;
                A[0] += R(1);
                A[4] += R(1);
                A[8] += R(1);
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        Fo[r + 3 * c] = A[r] * Fi[3 * c] + A[r + 3] * Fi[3 * c + 1] + A[r + 6] * Fi[3 * c + 2];
            }
            const int mat = (int)(idw >> 28);
            const MaterialDev<R>& M = sc->mat[mat];
            const R g_old = c_old * c_old * M.one_minus_theta + M.theta;
            const R alpha_in = w2.v[1], psi_in = w2.v[2];
            StressOut<R> so;
            constitutive_update<R, R, kAnyModel>(M, V0, dx, Fo, g_old, alpha_in, c_new, psi_in, so);
            if (fallback && so.smin_over_smax < ratio) {
                // FP64 SVD + return map for ill-conditioned F
                double Fd[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) Fd[q] = (double)Fo[q];
                StressOut<double> sd;
                constitutive_update<double, double, kAnyModel>(sc64->mat[mat], (double)V0, sc64->dx, Fd, (double)g_old, (double)alpha_in,
                                                 (double)c_new, (double)psi_in, sd);
#pragma unroll
                for (int q = 0; q < 9; ++q) so.F[q] = (R)sd.F[q];
#pragma unroll
                for (int q = 0; q < 6; ++q) so.sigma[q] = (R)sd.sigma[q];
                so.alpha = (R)sd.alpha;
                so.psi = (R)sd.psi;
                so.FP = (R)sd.FP;
                so.vol = (R)sd.vol;
                so.svd_ok = sd.svd_ok;
            }
            if (!so.svd_ok) flags |= GMPM_FLAG_SVD_NOCONVERGE;
            const R L0 = M.length_scale;
            const R qs = R(4) * L0 * L0 * so.vol;
#pragma unroll
            for (int a = 0; a < 3; ++a) aux.q[a][slot] = qs * gc[a];
#pragma unroll
            for (int q = 0; q < 9; ++q) finite = finite && isfinite(so.F[q]);
            out.fw[0][slot] = Word4<R>{{so.F[0], so.F[1], so.F[2], so.F[3]}};
            out.fw[1][slot] = Word4<R>{{so.F[4], so.F[5], so.F[6], so.F[7]}};
            out.fw[2][slot] = Word4<R>{{so.F[8], so.alpha, so.psi, R(0)}};
#pragma unroll
            for (int q = 0; q < 6; ++q) aux.sigma[q][slot] = so.sigma[q];
            aux.vol[slot] = so.vol;
            aux.FP[slot] = so.FP;
            if (!finite) flags |= GMPM_FLAG_NONFINITE;
        }
    }
    cp_async_wait_all();
    if (flags) raise_flag(cnt, flags);
    if (sc->adaptive_dt) {
        for (int off = 16; off > 0; off >>= 1) v2max = fmax(v2max, __shfl_xor_sync(0xffffffffu, v2max, off));
        if ((threadIdx.x & 31) == 0 && v2max > 0.0)
            atomicMax(&cnt->vmax2_bits, (unsigned long long)__double_as_longlong(v2max));
    }
}

// Advance the device clock after the substep's last reader of dt (G2P) and,
// in adaptive mode, set the next substep's dt from the maximum particle speed
// of this G2P: dt = min(dt_max, cfl dx / v_max) (MPMSimulator::computeDt,
// Simulator.cpp:200-225, on the device instead of through a host read).
template <typename R, bool kAnyModel, bool kFallback>
__global__ void __launch_bounds__(kG2PUnit, sizeof(R) == 4 ? kG2PMinBlocks : 1)
    k_g2p(const SceneDev<R>* __restrict__ sc, const SceneDev<double>* __restrict__ sc64, PState<R> in,
          PState<R> out, PAux<R> aux, BinDev bin, const R* __restrict__ nodes, Counters* cnt) {
    g2p_body<R, kAnyModel, kFallback>(own_blocks(), sc, sc64, in, out, aux, bin, nodes, cnt);
}

template <typename R>
__device__ __forceinline__ void advance_time_body(Counters* cnt, SceneDev<R>* sc, SceneDev<double>* sc64) {
    cnt->time += sc64->dt;
    cnt->substeps += 1;
    if (sc64->adaptive_dt) {
        const double vmax = sqrt(__longlong_as_double((long long)cnt->vmax2_bits));
        double dt = sc64->dt_max;
        if (vmax > 0 && sc64->cfl_dx / vmax < sc64->dt_max) dt = sc64->cfl_dx / vmax;
        sc64->dt = dt;
        sc->dt = (R)dt;
        cnt->vmax2_bits = 0ull;
    }
}

template <typename R>
__global__ void k_advance_time(Counters* cnt, SceneDev<R>* sc, SceneDev<double>* sc64) {
    advance_time_body<R>(cnt, sc, sc64);
}

// Batched launches: the same bodies for the scene that owns this CTA.  The
// FP64 fallback reads the scene's FP64 block only in the form with it.
template <typename R, bool kAnyModel, bool kFallback>
__global__ void __launch_bounds__(kG2PUnit, sizeof(R) == 4 ? kG2PMinBlocks : 1)
    k_batch_g2p(const SceneArgs<R>* __restrict__ A, const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    g2p_body<R, kAnyModel, kFallback>(vb, a.sc, kFallback ? a.sc64 : nullptr, a.in, a.out, a.aux, a.bin,
                                      reinterpret_cast<const R*>(a.grid.nodes), a.cnt);
}

template <typename R>
__global__ void k_batch_clock(const SceneArgs<R>* __restrict__ A, const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    if (threadIdx.x == 0)
        advance_time_body<R>(a.cnt, const_cast<SceneDev<R>*>(a.sc), const_cast<SceneDev<double>*>(a.sc64));
}

template <typename R>
cudaError_t prepare_g2p() {
    const int smem = (int)sizeof(G2PShared<R>);
    const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaFuncSetAttribute(k_g2p<R, false, false>, attr, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_g2p<R, true, false>, attr, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch_g2p<R, false, false>, attr, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch_g2p<R, true, false>, attr, smem);
    if constexpr (sizeof(R) == 4) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_g2p<R, false, true>, attr, smem);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_g2p<R, true, true>, attr, smem);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch_g2p<R, false, true>, attr, smem);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch_g2p<R, true, true>, attr, smem);
    }
    return e;
}

template <typename R>
cudaError_t launch_batch_g2p(const SceneArgs<R>* A, const BatchPlan& P, cudaStream_t s) {
    const dim3 grid((unsigned)P.total[BM_G2P]), block(kG2PUnit);
    const size_t smem = sizeof(G2PShared<R>);
    const int ns = P.n_scenes;
    const int32_t* st = P.start[BM_G2P];
    cudaError_t e;
    const bool fb = sizeof(R) == 4 && P.fallback;
    if (P.other_models)
        e = fb ? launch_kernel(k_batch_g2p<R, true, (sizeof(R) == 4)>, grid, block, smem, s, A, st, ns)
               : launch_kernel(k_batch_g2p<R, true, false>, grid, block, smem, s, A, st, ns);
    else
        e = fb ? launch_kernel(k_batch_g2p<R, false, (sizeof(R) == 4)>, grid, block, smem, s, A, st, ns)
               : launch_kernel(k_batch_g2p<R, false, false>, grid, block, smem, s, A, st, ns);
    if (e == cudaSuccess)
        e = launch_kernel(k_batch_clock<R>, dim3((unsigned)P.total[BM_ONE]), dim3(32), 0, s, A, P.start[BM_ONE], ns);
    return e;
}
template cudaError_t launch_batch_g2p<float>(const SceneArgs<float>*, const BatchPlan&, cudaStream_t);
template cudaError_t launch_batch_g2p<double>(const SceneArgs<double>*, const BatchPlan&, cudaStream_t);
template cudaError_t prepare_g2p<float>();
template cudaError_t prepare_g2p<double>();

template <typename R>
cudaError_t launch_g2p(const SceneDev<R>* sc, const SceneDev<double>* sc64, const SceneDev<double>* fallback64,
                       const PState<R>& in, const PState<R>& out, const PAux<R>& aux, BinDev bin, GridDev grid,
                       Counters* cnt, LaunchCfg cfg, cudaStream_t stream) {
    const int per_sm = sizeof(R) == 4 ? kG2PMinBlocks : 1;
    const int64_t units = (bin.n + kG2PUnit - 1) / kG2PUnit;
    const int ctas = (int)std::max<int64_t>(1, std::min<int64_t>(units, (int64_t)cfg.num_sms * per_sm));
    const R* nodes = reinterpret_cast<const R*>(grid.nodes);
    const size_t smem = sizeof(G2PShared<R>);
    // FP64 state needs no FP64 fallback; FP32 launches the fallback form only where the scene has it
    const bool fb = sizeof(R) == 4 && fallback64 != nullptr;
    if (cfg.other_models) {
        if (fb)
            k_g2p<R, true, (sizeof(R) == 4)><<<ctas, kG2PUnit, smem, stream>>>(sc, fallback64, in, out, aux, bin, nodes, cnt);
        else
            k_g2p<R, true, false><<<ctas, kG2PUnit, smem, stream>>>(sc, fallback64, in, out, aux, bin, nodes, cnt);
    } else {
        if (fb)
            k_g2p<R, false, (sizeof(R) == 4)><<<ctas, kG2PUnit, smem, stream>>>(sc, fallback64, in, out, aux, bin, nodes, cnt);
        else
            k_g2p<R, false, false><<<ctas, kG2PUnit, smem, stream>>>(sc, fallback64, in, out, aux, bin, nodes, cnt);
    }
    k_advance_time<R><<<1, 1, 0, stream>>>(cnt, const_cast<SceneDev<R>*>(sc), const_cast<SceneDev<double>*>(sc64));
    return cudaGetLastError();
}

template cudaError_t launch_g2p<float>(const SceneDev<float>*, const SceneDev<double>*, const SceneDev<double>*,
                                       const PState<float>&, const PState<float>&, const PAux<float>&, BinDev,
                                       GridDev, Counters*, LaunchCfg, cudaStream_t);
template cudaError_t launch_g2p<double>(const SceneDev<double>*, const SceneDev<double>*, const SceneDev<double>*,
                                        const PState<double>&, const PState<double>&, const PAux<double>&, BinDev,
                                        GridDev, Counters*, LaunchCfg, cudaStream_t);

}  // namespace gmpm
