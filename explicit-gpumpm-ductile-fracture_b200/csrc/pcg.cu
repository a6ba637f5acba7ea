// Implicit phase field: the reference's Jacobi-preconditioned CG solve of
//     (D + M K) c = M_L (c_grid / dt + M)
// on the tagged grid nodes (ExplicitTimeIntegrator.cu:909-972), with
//     D_i   = sum_p V w_ip (FP M + 1/dt)                 (preConditionP2G_APIC)
//     (K x)_i = sum_p grad w_ip . col_p,
//     col_p = 4 L0^2 V_p sum_j grad w_jp x_j             (AxG2P_APIC, AxP2G_APIC)
// All vectors and scalars are FP64, as in the reference.  The scalars of the
// iteration (alpha, rho, rate, the residual norm) stay on the device: every
// kernel of an iteration first checks the solve's `done` flag, so iterations
// launched after convergence cost only their launch.
//
// Determinism: dot products are partial sums over runs of 128 entries in a
// fixed tree order, combined in a fixed order (by max instead of a sum when
// the reference's getDotProduct quirk is selected, :727-743), and K x is
// summed per cell z-column and gathered per node in a fixed order, so runs
// are bitwise reproducible.
#include <cstdint>

#include "kernels.h"

namespace gmpm {

constexpr int kPcgBlock = 128;     // vector entries per partial sum (2 grid pages)
constexpr int kPcgScalarThreads = 1024;
constexpr int kPcgColThreads = 256;
constexpr int kPcgKxWarps = 8;     // two cell z-columns of a page each
constexpr int kPcgKxCols = 16 / kPcgKxWarps;
constexpr int kPcgKxThreads = 32 * kPcgKxWarps;
constexpr int kPcgKxChunk = 512;   // particles staged per pass of a page
constexpr int kKxRec = 11;         // staged per particle: xp0, xp1, wz[3], gz[3], col[3]

// ---- helpers -----------------------------------------------------------------

// quadratic B-spline weight and gradient of stencil node k (0..2) along one
// axis, xp relative to the base node (AxG2P_APIC, G2PKernal.cu:1063-1083)
__device__ __forceinline__ void bspline_k(double xp, double inv_dx, int k, double& w, double& g) {
    const double d0 = xp * inv_dx;
    if (k == 0) {
        const double z = 1.5 - d0;
        w = 0.5 * z * z;
        g = -z * inv_dx;
    } else if (k == 1) {
        const double d = d0 - 1.0;
        w = 0.75 - d * d;
        g = -d * 2.0 * inv_dx;
    } else {
        const double z = 1.5 - (1.0 - (d0 - 1.0));
        w = 0.5 * z * z;
        g = z * inv_dx;
    }
}

// Block tree sum (fixed order) of one value per thread.
template <int T>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < T / 32 ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;  // valid in thread 0
}

template <int T>
__device__ __forceinline__ double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x < 32) {
        r = threadIdx.x < T / 32 ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;
}

__device__ __forceinline__ int pcg_entries(const Counters* cnt, const BinDev& bin) {
    return min(cnt->n_grid_blocks, bin.ng_cap) * 64;
}

// Combine partial sums [0, n) in a fixed order: sum, or max (quirk).
__device__ double combine_partials(const double* part, int n, bool use_max, double* sh) {
    double acc = 0.0;
    bool any = false;
    for (int i = threadIdx.x; i < n; i += kPcgScalarThreads) {
        const double v = part[i];
        acc = use_max ? (any ? fmax(acc, v) : v) : acc + v;
        any = true;
    }
    if (use_max) {
        if (!any) acc = -1.0 / 0.0;
        return block_max<kPcgScalarThreads>(acc, sh);
    }
    return block_sum<kPcgScalarThreads>(acc, sh);
}

// ---- kernels -----------------------------------------------------------------

// partial sums of a[i] b[i] over runs of 128 entries
__global__ void __launch_bounds__(kPcgBlock)
    k_pcg_dot(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ part, BinDev bin,
              const Counters* __restrict__ cnt) {
    __shared__ double sh[32];
    const int N = pcg_entries(cnt, bin);
    const int nparts = (N + kPcgBlock - 1) / kPcgBlock;
    for (int blk = blockIdx.x; blk < nparts; blk += gridDim.x) {
        const int i = blk * kPcgBlock + threadIdx.x;
        const double v = i < N ? a[i] * b[i] : 0.0;
        const double s = block_sum<kPcgBlock>(v, sh);
        if (threadIdx.x == 0) part[blk] = s;
    }
}

__global__ void __launch_bounds__(kPcgScalarThreads)
    k_pcg_start(PcgDev P, BinDev bin, Counters* cnt, int max_combine) {
    __shared__ double sh[32];
    const int N = pcg_entries(cnt, bin);
    const double rho = combine_partials(P.part, (N + kPcgBlock - 1) / kPcgBlock, max_combine != 0, sh);
    if (threadIdx.x == 0) {
        P.scal->rho_old = rho;
        P.scal->alpha = P.scal->rate = P.scal->norm = 0.0;
        P.scal->done = (N == 0);
        P.scal->blowup = 0;
        P.scal->iterations = 0;
    }
}

// col_p = 4 L0^2 V_p sum_j grad w_jp s_j (AxG2P_APIC, G2PKernal.cu:1006-1123):
// one CTA per particle page with the page's 6x6x6 window of s staged.
template <typename R>
__global__ void __launch_bounds__(kPcgColThreads)
    k_pcg_col(const SceneDev<R>* __restrict__ sc, PState<R> st, PAux<R> aux, BinDev bin, PcgDev P,
              const Counters* __restrict__ cnt) {
    if (P.scal->done) return;
    __shared__ double win[kWindowNodes];
    const int nb = min(cnt->n_blocks, bin.nb_cap);
    const double dx = sc->dx_d, inv_dx = sc->inv_dx_d;
    // col of the particle in `slot` (previous slot o, cell, position x, volume, id)
    auto particle = [&](int slot, int o, uint32_t cell, const R* x, R vol, uint32_t idw, int bx, int by, int bz) {
        const int li = (int)(cell >> 4), lj = (int)((cell >> 2) & 3), lk = (int)(cell & 3);
        const double xp[3] = {(double)x[0] - (double)(4 * bx + li) * dx, (double)x[1] - (double)(4 * by + lj) * dx,
                              (double)x[2] - (double)(4 * bz + lk) * dx};
        double w[3][3], gr[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int k = 0; k < 3; ++k) bspline_k(xp[a], inv_dx, k, w[a][k], gr[a][k]);
        double col[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const double xn = win[(li + i) * 36 + (lj + j) * 6 + (lk + k)];
                    col[0] += gr[0][i] * w[1][j] * w[2][k] * xn;
                    col[1] += w[0][i] * gr[1][j] * w[2][k] * xn;
                    col[2] += w[0][i] * w[1][j] * gr[2][k] * xn;
                }
        const double L0 = (double)sc->mat[idw >> 28].length_scale;
        const double para = (double)vol * 4.0 * L0 * L0;
#pragma unroll
        for (int a = 0; a < 3; ++a) P.col[(int64_t)a * P.n + slot] = col[a] * para;
        (void)o;
    };
    for (int b = blockIdx.x; b < nb; b += gridDim.x) {
        // The page's bounds and this thread's first particle are loaded before
        // the window, so the two chains of dependent loads overlap.
        const int s0 = bin.cell_start[(int64_t)b * 64], s1 = bin.cell_start[(int64_t)b * 64 + 64];
        int bx, by, bz;
        page_coords(bin.block_keys[b], bx, by, bz);
        const int slot0 = s0 + (int)threadIdx.x;
        int o0 = 0;
        uint32_t cell0 = 0, id0 = 0;
        R x0[3] = {R(0), R(0), R(0)}, vol0 = R(0);
        if (slot0 < s1) {
            o0 = bin.perm[slot0];
            cell0 = bin.keys_sorted[slot0] & 63u;
#pragma unroll
            for (int a = 0; a < 3; ++a) x0[a] = st.x[a][o0];
            vol0 = aux.vol[o0];
            id0 = st.id[o0];
        }
        __syncthreads();
        for (int w = threadIdx.x; w < kWindowNodes; w += kPcgColThreads) {
            const int a = w / 36, bb = (w / 6) % 6, cc = w % 6;
            const int d = ((a >> 2) << 2) | ((bb >> 2) << 1) | (cc >> 2);
            const int g = bin.adj[(int64_t)b * 8 + d];
            win[w] = g < 0 ? 0.0 : P.s[(int64_t)g * 64 + (a & 3) * 16 + (bb & 3) * 4 + (cc & 3)];
        }
        __syncthreads();
        if (slot0 < s1) particle(slot0, o0, cell0, x0, vol0, id0, bx, by, bz);
        for (int slot = slot0 + kPcgColThreads; slot < s1; slot += kPcgColThreads) {
            const int o = bin.perm[slot];
            const R x[3] = {st.x[0][o], st.x[1][o], st.x[2][o]};
            particle(slot, o, bin.keys_sorted[slot] & 63u, x, aux.vol[o], st.id[o], bx, by, bz);
        }
    }
}

// x or y B-spline piece of stencil node k for one lane, branch-free:
// w = a z^2 + b and dw/dx = c z with z = xp/dx - shift.
struct KxPiece {
    double shift, a, b, c;
    __device__ void init(int k, double inv_dx) {
        shift = k == 0 ? 1.5 : (k == 1 ? 1.0 : 0.5);
        a = k == 1 ? -1.0 : 0.5;
        b = k == 1 ? 0.75 : 0.0;
        c = (k == 1 ? -2.0 : 1.0) * inv_dx;
    }
    __device__ __forceinline__ void eval(double xp, double inv_dx, double& w, double& g) const {
        const double z = xp * inv_dx - shift;
        w = a * (z * z) + b;
        g = c * z;
    }
};

// One particle of cell z-index CZ into the lane's six z-node sums:
// grad w . col = wz (gx wy c0 + wx gy c1) + gz (wx wy c2).
template <int CZ>
__device__ __forceinline__ void kx_accumulate(const double* __restrict__ r, const KxPiece& px, const KxPiece& py,
                                              double inv_dx, double* acc) {
    double wx, gx, wy, gy;
    px.eval(r[0], inv_dx, wx, gx);
    py.eval(r[1], inv_dx, wy, gy);
    const double u = gx * wy * r[8] + wx * gy * r[9];
    const double v = wx * wy * r[10];
#pragma unroll
    for (int k = 0; k < 3; ++k) acc[CZ + k] += r[2 + k] * u + r[5 + k] * v;
}

template <int CZ>
__device__ __forceinline__ void kx_cell(const double* __restrict__ recs, const int* __restrict__ cs, int cb, int c0,
                                        int c1, int sub, const KxPiece& px, const KxPiece& py, double inv_dx,
                                        double* acc) {
    const int lo = max(cs[cb + CZ], c0) - c0, hi = min(cs[cb + CZ + 1], c1) - c0;
#pragma unroll 2
    for (int p = lo + sub; p < hi; p += 3) kx_accumulate<CZ>(recs + (size_t)p * kKxRec, px, py, inv_dx, acc);
}

// Page tile of K s (AxP2G_APIC): window node (a, b, c) sums grad w . col over
// the particles whose stencil covers it.  As in the P2G, per cell z-column
// (cx, cy): eight warps own two columns each (small CTAs, four per SM, keep
// more pages in flight); lane (sub, i, j) = particle stream sub (the warp takes
// three particles of a cell per step) x stencil column (i, j), with the sums
// of window nodes (cx+i, cy+j, 0..5) in registers.  At the page's end the
// three streams of a stencil column are added in fixed order, and each window
// node gathers its (at most 9) columns in fixed order, compensated, so runs
// are bitwise reproducible.
template <typename R>
__global__ void __launch_bounds__(kPcgKxThreads, 4)
    k_pcg_kx(const SceneDev<R>* __restrict__ sc, PState<R> st, BinDev bin, PcgDev P, double* __restrict__ tile,
             const Counters* __restrict__ cnt) {
    if (P.scal->done) return;
    __shared__ double recs[kPcgKxChunk * kKxRec];  // staged particles; the column sums at a page's end
    __shared__ int cstart[65];
    static_assert(16 * 9 * 6 <= kPcgKxChunk * kKxRec, "column sums fit the staging buffer");
    const int nb = min(cnt->n_blocks, bin.nb_cap);
    const double dx = sc->dx_d, inv_dx = sc->inv_dx_d;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int le = lane < 27 ? lane : lane - 27;  // lanes 27..31 shadow lanes 0..4 and never write
    const int sub = le / 9, col = le - sub * 9;
    const int ci = col / 3, cj = col - ci * 3;
    // column h of warp w: index w + 8 h, cx its high bits, cy rotated by cx
    // (the warps of a scheduler hold one column of every cx and cy)
    int cpos[kPcgKxCols], cb[kPcgKxCols];
#pragma unroll
    for (int h = 0; h < kPcgKxCols; ++h) {
        const int cidx = warp + h * kPcgKxWarps;
        const int cx = cidx >> 2, cy = ((cidx & 3) - cx) & 3;
        cpos[h] = cx * 4 + cy;
        cb[h] = cx * 16 + cy * 4;
    }
    KxPiece px, py;
    px.init(ci, inv_dx);
    py.init(cj, inv_dx);
    for (int b = blockIdx.x; b < nb; b += gridDim.x) {
        __syncthreads();
        for (int q = t; q < 65; q += kPcgKxThreads) cstart[q] = bin.cell_start[(int64_t)b * 64 + q];
        int bx, by, bz;
        page_coords(bin.block_keys[b], bx, by, bz);
        __syncthreads();
        double acc[kPcgKxCols][6];
#pragma unroll
        for (int h = 0; h < kPcgKxCols; ++h)
#pragma unroll
            for (int z = 0; z < 6; ++z) acc[h][z] = 0.0;
        for (int c0 = cstart[0]; c0 < cstart[64]; c0 += kPcgKxChunk) {
            const int c1 = min(cstart[64], c0 + kPcgKxChunk);
            __syncthreads();
            for (int slot = c0 + t; slot < c1; slot += kPcgKxThreads) {
                const int o = bin.perm[slot];
                const uint32_t cell = bin.keys_sorted[slot] & 63u;
                const int base[3] = {4 * bx + (int)(cell >> 4), 4 * by + (int)((cell >> 2) & 3),
                                     4 * bz + (int)(cell & 3)};
                double* r = recs + (size_t)(slot - c0) * kKxRec;
                r[0] = (double)st.x[0][o] - (double)base[0] * dx;
                r[1] = (double)st.x[1][o] - (double)base[1] * dx;
                const double xp2 = (double)st.x[2][o] - (double)base[2] * dx;
#pragma unroll
                for (int k = 0; k < 3; ++k) bspline_k(xp2, inv_dx, k, r[2 + k], r[5 + k]);
#pragma unroll
                for (int a = 0; a < 3; ++a) r[8 + a] = P.col[(int64_t)a * P.n + slot];
            }
            __syncthreads();
#pragma unroll
            for (int h = 0; h < kPcgKxCols; ++h) {
                kx_cell<0>(recs, cstart, cb[h], c0, c1, sub, px, py, inv_dx, acc[h]);
                kx_cell<1>(recs, cstart, cb[h], c0, c1, sub, px, py, inv_dx, acc[h]);
                kx_cell<2>(recs, cstart, cb[h], c0, c1, sub, px, py, inv_dx, acc[h]);
                kx_cell<3>(recs, cstart, cb[h], c0, c1, sub, px, py, inv_dx, acc[h]);
            }
        }
        // the three particle streams of a stencil column, in fixed order
#pragma unroll
        for (int h = 0; h < kPcgKxCols; ++h)
#pragma unroll
            for (int z = 0; z < 6; ++z) {
                const double v1 = __shfl_sync(0xffffffffu, acc[h][z], (lane + 9) & 31);
                const double v2 = __shfl_sync(0xffffffffu, acc[h][z], (lane + 18) & 31);
                acc[h][z] = (acc[h][z] + v1) + v2;
            }
        __syncthreads();  // every warp is past its sweep: the staging buffer is free
        double* colsum = recs;  // [column 4 cx + cy][stencil column][z]
        if (lane < 9) {
#pragma unroll
            for (int h = 0; h < kPcgKxCols; ++h)
#pragma unroll
                for (int z = 0; z < 6; ++z) colsum[(cpos[h] * 9 + col) * 6 + z] = acc[h][z];
        }
        __syncthreads();
        if (t < kWindowNodes) {
            const int na = t / 36, nbb = (t / 6) % 6, nc = t % 6;
            double sum = 0.0, comp = 0.0;
            for (int cx = max(0, na - 2); cx <= min(3, na); ++cx)
                for (int cy = max(0, nbb - 2); cy <= min(3, nbb); ++cy)
                    kahan_add(sum, comp, colsum[((cx * 4 + cy) * 9 + (na - cx) * 3 + (nbb - cy)) * 6 + nc]);
            tile[(int64_t)b * kWindowNodes + t] = sum;
        }
    }
}

// q = D s + M K s on tagged nodes (K s: the 8 overlapping page tiles in slot
// order); partial sums of s . q
__global__ void __launch_bounds__(kPcgBlock)
    k_pcg_q(BinDev bin, PcgDev P, const double* __restrict__ tile, const Counters* __restrict__ cnt,
            double mobility) {
    if (P.scal->done) return;
    __shared__ double sh[32];
    const int N = pcg_entries(cnt, bin);
    const int nparts = (N + kPcgBlock - 1) / kPcgBlock;
    const int node = threadIdx.x & 63;
    const int ci = node >> 4, cj = (node >> 2) & 3, ck = node & 3;
    for (int blk = blockIdx.x; blk < nparts; blk += gridDim.x) {
        const int i = blk * kPcgBlock + threadIdx.x;
        double sq = 0.0;
        if (i < N) {
            const int g = i >> 6;
            double kx = 0.0;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const int a = 4 * (d >> 2) + ci, b = 4 * ((d >> 1) & 1) + cj, c = 4 * (d & 1) + ck;
                if (a >= 6 || b >= 6 || c >= 6) continue;
                const int src = bin.grid_src[g * 8 + d];
                if (src < 0) continue;
                kx += tile[(int64_t)src * kWindowNodes + a * 36 + b * 6 + c];
            }
            const double q = P.tag[i] ? P.d[i] * P.s[i] + mobility * kx : 0.0;
            P.q[i] = q;
            sq = P.s[i] * q;
        }
        const double s = block_sum<kPcgBlock>(sq, sh);
        if (threadIdx.x == 0) P.part[blk] = s;
    }
}

__global__ void __launch_bounds__(kPcgScalarThreads)
    k_pcg_alpha(PcgDev P, BinDev bin, const Counters* __restrict__ cnt, int max_combine) {
    if (P.scal->done) return;
    __shared__ double sh[32];
    const int N = pcg_entries(cnt, bin);
    const double sq = combine_partials(P.part, (N + kPcgBlock - 1) / kPcgBlock, max_combine != 0, sh);
    if (threadIdx.x == 0) P.scal->alpha = P.scal->rho_old / sq;
}

// x += alpha s, r -= alpha q, mr = r / D (precondition_subd) on tagged nodes;
// partial max r^2 and partial sums of r . mr
__global__ void __launch_bounds__(kPcgBlock)
    k_pcg_update(BinDev bin, PcgDev P, const Counters* __restrict__ cnt) {
    if (P.scal->done) return;
    __shared__ double sh[32];
    const int N = pcg_entries(cnt, bin);
    const int nparts = (N + kPcgBlock - 1) / kPcgBlock;
    const double alpha = P.scal->alpha;
    double* pmax = P.part + P.nparts_cap;
    double* pdot = P.part + 2 * P.nparts_cap;
    for (int blk = blockIdx.x; blk < nparts; blk += gridDim.x) {
        const int i = blk * kPcgBlock + threadIdx.x;
        double r2 = 0.0, rm = 0.0;
        if (i < N) {
            double r = P.r[i], mr = P.mr[i];
            if (P.tag[i]) {
                P.x[i] += P.s[i] * alpha;
                r = r - P.q[i] * alpha;
                P.r[i] = r;
                const double dg = P.d[i];
                if (fabs(dg) >= 1e-30) {
                    mr = r / dg;
                    P.mr[i] = mr;
                }
            }
            r2 = r * r;
            rm = r * mr;
        }
        const double m = block_max<kPcgBlock>(r2, sh);
        const double s = block_sum<kPcgBlock>(rm, sh);
        if (threadIdx.x == 0) {
            pmax[blk] = m;
            pdot[blk] = s;
        }
    }
}

// residual norm, convergence, rho and the direction update rate
__global__ void __launch_bounds__(kPcgScalarThreads)
    k_pcg_rho(PcgDev P, BinDev bin, const Counters* __restrict__ cnt, int max_combine, double tol) {
    if (P.scal->done) return;
    __shared__ double sh[32];
    const int N = pcg_entries(cnt, bin);
    const int nparts = (N + kPcgBlock - 1) / kPcgBlock;
    double m = 0.0;
    for (int i = threadIdx.x; i < nparts; i += kPcgScalarThreads) m = fmax(m, P.part[P.nparts_cap + i]);
    const double norm = sqrt(block_max<kPcgScalarThreads>(m, sh));
    const double rho = combine_partials(P.part + 2 * P.nparts_cap, nparts, max_combine != 0, sh);
    if (threadIdx.x == 0) {
        PcgScalars& S = *P.scal;
        S.iterations += 1;
        S.norm = norm;
        if (norm < tol) {
            S.done = 1;
        } else if (S.rho_old == 0.0) {
            S.blowup = 1;
            S.done = 1;
        } else {
            S.rate = rho / S.rho_old;
            S.rho_old = rho;
        }
    }
}

// s = s rate + mr on tagged nodes (cal_grid_r_vad_kernal)
__global__ void __launch_bounds__(kPcgBlock) k_pcg_sdir(BinDev bin, PcgDev P, const Counters* __restrict__ cnt) {
    if (P.scal->done) return;
    const int N = pcg_entries(cnt, bin);
    const double rate = P.scal->rate;
    for (int i = blockIdx.x * kPcgBlock + threadIdx.x; i < N; i += gridDim.x * kPcgBlock)
        if (P.tag[i]) P.s[i] = P.s[i] * rate + P.mr[i];
}

// dc = x - c_grid and c_new = x on tagged nodes (update_grid_phase, :632-642);
// x = 1e20 everywhere after a breakdown (rho_old == 0)
template <typename R>
__global__ void k_pcg_finish(BinDev bin, PcgDev P, R* __restrict__ nodes, Counters* cnt) {
    const int N = pcg_entries(cnt, bin);
    const bool blow = P.scal->blowup != 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        if (!P.tag[i]) continue;
        const double x = blow ? 1e20 : P.x[i];
        R* nd = nodes + (int64_t)(i >> 6) * kGridChannels * 64 + (i & 63);
        nd[GC_DC * 64] = (R)(x - P.cg[i]);
        nd[GC_CN * 64] = (R)x;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt->pcg_iterations = P.scal->iterations;
}

// ---- launchers ---------------------------------------------------------------

namespace {
int pcg_grid_blocks(const BinDev& bin, const LaunchCfg& cfg) {
    const int nparts = (bin.ng_cap * 64 + kPcgBlock - 1) / kPcgBlock;
    return max(1, min(nparts, cfg.num_sms * 16));
}
}  // namespace

template <typename R>
cudaError_t launch_pcg_init(const SceneDev<R>* sc, BinDev bin, GridDev grid, Counters* cnt, LaunchCfg cfg,
                            cudaStream_t stream) {
    const PcgDev& P = grid.pcg;
    k_pcg_dot<<<pcg_grid_blocks(bin, cfg), kPcgBlock, 0, stream>>>(P.r, P.mr, P.part, bin, cnt);
    k_pcg_start<<<1, kPcgScalarThreads, 0, stream>>>(P, bin, cnt, cfg.pcg_max_combine);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_pcg_iteration(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, BinDev bin,
                                 GridDev grid, Counters* cnt, LaunchCfg cfg, cudaStream_t stream) {
    const PcgDev& P = grid.pcg;
    double* tile = reinterpret_cast<double*>(grid.tile);
    const int pages = max(1, min(bin.nb_cap, cfg.num_sms * 4));
    const int gb = pcg_grid_blocks(bin, cfg);
    k_pcg_col<R><<<pages, kPcgColThreads, 0, stream>>>(sc, st, aux, bin, P, cnt);
    k_pcg_kx<R><<<max(1, min(bin.nb_cap, cfg.num_sms * 8)), kPcgKxThreads, 0, stream>>>(sc, st, bin, P, tile, cnt);
    k_pcg_q<<<gb, kPcgBlock, 0, stream>>>(bin, P, tile, cnt, cfg.pcg_mobility);
    k_pcg_alpha<<<1, kPcgScalarThreads, 0, stream>>>(P, bin, cnt, cfg.pcg_max_combine);
    k_pcg_update<<<gb, kPcgBlock, 0, stream>>>(bin, P, cnt);
    k_pcg_rho<<<1, kPcgScalarThreads, 0, stream>>>(P, bin, cnt, cfg.pcg_max_combine, cfg.pcg_tolerance);
    k_pcg_sdir<<<gb, kPcgBlock, 0, stream>>>(bin, P, cnt);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_pcg_finish(const SceneDev<R>* sc, BinDev bin, GridDev grid, Counters* cnt, LaunchCfg cfg,
                              cudaStream_t stream) {
    k_pcg_finish<R><<<pcg_grid_blocks(bin, cfg), kPcgBlock, 0, stream>>>(bin, grid.pcg,
                                                                         reinterpret_cast<R*>(grid.nodes), cnt);
    return cudaGetLastError();
}

#define GMPM_PCG_INST(R)                                                                                            \
    template cudaError_t launch_pcg_init<R>(const SceneDev<R>*, BinDev, GridDev, Counters*, LaunchCfg,              \
                                            cudaStream_t);                                                         \
    template cudaError_t launch_pcg_iteration<R>(const SceneDev<R>*, const PState<R>&, const PAux<R>&, BinDev,      \
                                                 GridDev, Counters*, LaunchCfg, cudaStream_t);                      \
    template cudaError_t launch_pcg_finish<R>(const SceneDev<R>*, BinDev, GridDev, Counters*, LaunchCfg, cudaStream_t);
GMPM_PCG_INST(float)
GMPM_PCG_INST(double)

}  // namespace gmpm
