// G2P: grid-to-particle transfer (G2P_APIC, G2PKernal.cu:204-441) fused with
// the constitutive update that the reference runs at the start of the next
// substep (applyVonMises, ExplicitTimeIntegrator.cu:132-370) and with the
// phase-field gradient gather (AxG2P_APIC, G2PKernal.cu:1006-1123).
//
// One CTA per particle page: the page's 6x6x6 window of v, dc and c_new is
// staged in shared memory; one thread per particle then gathers its 3x3x3
// stencil, updates c (irreversibly), x, F = (I + dt grad v) F, the APIC matrix
// B, runs the SVD + Hencky return map + damage driving force, and writes the
// particle in the new sorted order.  Reading the previous order through perm
// and writing the new order is the reorder the reference does with gathers
// and D2D copies (Particle_kernal.cu:544-573, TimeIntegrator.cu:459-461).
#include <cstdint>

#include "constitutive.cuh"
#include "kernels.h"

namespace gmpm {

constexpr int kG2PThreads = 256;

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

template <typename R>
__global__ void __launch_bounds__(kG2PThreads, sizeof(R) == 4 ? 2 : 1)
    k_g2p(const SceneDev<R>* __restrict__ sc, const SceneDev<double>* __restrict__ sc64, PState<R> in,
          PState<R> out, PAux<R> aux, BinDev bin, const R* __restrict__ nodes, Counters* cnt) {
    // window of the page: (v0, v1, v2, dc) per node as one 16-byte group, c_new apart
    __shared__ __align__(16) R win4[kWindowNodes][4];
    __shared__ R wincn[kWindowNodes];
    const int nb = min(cnt->n_blocks, bin.nb_cap);
    const R dx = sc->dx, inv_dx = sc->inv_dx, dt = sc->dt, V0 = sc->V0;
    const bool fallback = sc->fp64_svd_fallback && sc64 != nullptr;
    const R ratio = sc->svd_fallback_ratio;
    unsigned int flags = 0;

    for (int b = blockIdx.x; b < nb; b += gridDim.x) {
        int bx, by, bz;
        page_coords(bin.block_keys[b], bx, by, bz);
        const int32_t* adj = bin.adj + (int64_t)b * 8;
        for (int w = threadIdx.x; w < kGridChannels * kWindowNodes; w += kG2PThreads) {
            const int ch = w / kWindowNodes;
            const int node = w - ch * kWindowNodes;
            const int a = node / 36, bb = (node / 6) % 6, cc = node % 6;
            const int d = ((a >> 2) << 2) | ((bb >> 2) << 1) | (cc >> 2);
            const int g = adj[d];
            const R val = (g >= 0) ? nodes[(int64_t)g * kGridChannels * 64 + ch * 64 + (a & 3) * 16 + (bb & 3) * 4 +
                                           (cc & 3)]
                                   : R(0);
            if (ch < 4)
                win4[node][ch] = val;
            else
                wincn[node] = val;
        }
        __syncthreads();
        const int bs = bin.cell_start[(int64_t)b * 64], be = bin.cell_start[(int64_t)b * 64 + 64];
        for (int slot = bs + threadIdx.x; slot < be; slot += kG2PThreads) {
            const int o = bin.perm[slot];
            const uint32_t cell = bin.keys_sorted[slot] & 63u;
            const int li = (int)(cell >> 4), lj = (int)((cell >> 2) & 3), lk = (int)(cell & 3);
            const R x[3] = {in.x[0][o], in.x[1][o], in.x[2][o]};
            const R xp[3] = {x[0] - R(4 * bx + li) * dx, x[1] - R(4 * by + lj) * dx, x[2] - R(4 * bz + lk) * dx};
            R wx[3], gx[3], wy[3], gy[3], wz[3], gz[3];
            bspline1d_g(xp[0], inv_dx, wx, gx);
            bspline1d_g(xp[1], inv_dx, wy, gy);
            bspline1d_g(xp[2], inv_dx, wz, gz);
            R vp[3] = {R(0), R(0), R(0)}, dcp = R(0);
            R gv[9], Bn[9], gc[3] = {R(0), R(0), R(0)};
#pragma unroll
            for (int q = 0; q < 9; ++q) gv[q] = Bn[q] = R(0);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const R d0 = R(i) * dx - xp[0];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const R d1 = R(j) * dx - xp[1];
                    const R wxy = wx[i] * wy[j], gxy0 = gx[i] * wy[j], gxy1 = wx[i] * gy[j];
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const R d2 = R(k) * dx - xp[2];
                        const int node = (li + i) * 36 + (lj + j) * 6 + (lk + k);
                        R nv[4];
                        if (sizeof(R) == 4) {
                            *reinterpret_cast<float4*>(nv) = *reinterpret_cast<const float4*>(&win4[node][0]);
                        } else {
                            *reinterpret_cast<double2*>(nv) = *reinterpret_cast<const double2*>(&win4[node][0]);
                            *reinterpret_cast<double2*>(nv + 2) = *reinterpret_cast<const double2*>(&win4[node][2]);
                        }
                        const R n0 = nv[0], n1 = nv[1], n2 = nv[2], ndc = nv[3], ncn = wincn[node];
                        const R w = wxy * wz[k];
                        const R wg[3] = {gxy0 * wz[k], gxy1 * wz[k], wxy * gz[k]};
                        vp[0] += w * n0;
                        vp[1] += w * n1;
                        vp[2] += w * n2;
                        dcp += w * ndc;
                        const R dd[3] = {d0, d1, d2};
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            gv[0 + 3 * c] += n0 * wg[c];
                            gv[1 + 3 * c] += n1 * wg[c];
                            gv[2 + 3 * c] += n2 * wg[c];
                            const R wd = w * dd[c];
                            Bn[0 + 3 * c] += n0 * wd;
                            Bn[1 + 3 * c] += n1 * wd;
                            Bn[2 + 3 * c] += n2 * wd;
                            gc[c] += wg[c] * ncn;
                        }
                    }
                }
            }
            // damage: irreversible (G2PKernal.cu:359-366)
            const R c_old = in.c[o];
            const R c_new = fmax(fmin(c_old, c_old + dcp), R(0));
            // Write the transfer results first so they are dead during the SVD.
            bool finite = true;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const R xn = x[a] + vp[a] * dt;
                out.x[a][slot] = xn;
                aux.v[a][slot] = vp[a];
                finite = finite && isfinite(xn);
            }
#pragma unroll
            for (int q = 0; q < 9; ++q) aux.B[q][slot] = Bn[q];
            out.c[slot] = c_new;
            out.m[slot] = in.m[o];
            const uint32_t idw = in.id[o];
            out.id[slot] = idw;
            // F <- (I + dt grad v) F  (G2PKernal.cu:372-404)
            R Fo[9];
            {
                R A[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) A[q] = gv[q] * dt;
                A[0] += R(1);
                A[4] += R(1);
                A[8] += R(1);
                R Fi[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) Fi[q] = in.F[q][o];
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        Fo[r + 3 * c] = A[r] * Fi[3 * c] + A[r + 3] * Fi[3 * c + 1] + A[r + 6] * Fi[3 * c + 2];
            }
            const int mat = (int)(idw >> 28);
            const MaterialDev<R>& M = sc->mat[mat];
            const R theta = M.theta;
            const R g_old = c_old * c_old * (R(1) - theta) + theta;
            StressOut<R> so;
            von_mises_update<R, R>(M, V0, Fo, g_old, in.alpha[o], c_new, in.psi[o], so);
            if (fallback && so.smin_over_smax < ratio) {
                // FP64 SVD + return map for ill-conditioned F
                double Fd[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) Fd[q] = (double)Fo[q];
                StressOut<double> sd;
                von_mises_update<double, double>(sc64->mat[mat], (double)V0, Fd, (double)g_old,
                                                 (double)in.alpha[o], (double)c_new, (double)in.psi[o], sd);
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
            for (int q = 0; q < 9; ++q) {
                out.F[q][slot] = so.F[q];
                finite = finite && isfinite(so.F[q]);
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) aux.sigma[q][slot] = so.sigma[q];
            out.alpha[slot] = so.alpha;
            out.psi[slot] = so.psi;
            aux.vol[slot] = so.vol;
            aux.FP[slot] = so.FP;
            if (!finite) flags |= GMPM_FLAG_NONFINITE;
        }
        __syncthreads();
    }
    if (flags) raise_flag(cnt, flags);
}

// Advance the device clock after the substep's last reader of it (the grid kernel).
__global__ void k_advance_time(Counters* cnt, const double* dt) {
    cnt->time += *dt;
    cnt->substeps += 1;
}

template <typename R>
cudaError_t prepare_g2p() {
    return cudaSuccess;
}
template cudaError_t prepare_g2p<float>();
template cudaError_t prepare_g2p<double>();

template <typename R>
cudaError_t launch_g2p(const SceneDev<R>* sc, const SceneDev<double>* sc64, const SceneDev<double>* fallback64,
                       const PState<R>& in, const PState<R>& out, const PAux<R>& aux, BinDev bin, GridDev grid,
                       Counters* cnt, LaunchCfg cfg, cudaStream_t stream) {
    const int ctas = max(1, min(bin.nb_cap, cfg.num_sms * 8));
    k_g2p<R><<<ctas, kG2PThreads, 0, stream>>>(sc, fallback64, in, out, aux, bin,
                                               reinterpret_cast<const R*>(grid.nodes), cnt);
    k_advance_time<<<1, 1, 0, stream>>>(cnt, &sc64->dt);
    return cudaGetLastError();
}

template cudaError_t launch_g2p<float>(const SceneDev<float>*, const SceneDev<double>*, const SceneDev<double>*,
                                       const PState<float>&, const PState<float>&, const PAux<float>&, BinDev,
                                       GridDev, Counters*, LaunchCfg, cudaStream_t);
template cudaError_t launch_g2p<double>(const SceneDev<double>*, const SceneDev<double>*, const SceneDev<double>*,
                                        const PState<double>&, const PState<double>&, const PAux<double>&, BinDev,
                                        GridDev, Counters*, LaunchCfg, cudaStream_t);

}  // namespace gmpm
