// Grid stage, one thread per node of every grid page (active pages and their
// "+" neighbours):
//   * fixed-order, compensated (Kahan) sum of the (up to 8) P2G page tiles
//     overlapping the page,
//   * undateGrid_kernal (TimeIntegrator.cu:63-111): c = C/W, v = p/m + g dt
//     (the force is already in p),
//   * explicit phase-field update replacing the reference's Jacobi-PCG solve
//     (ExplicitTimeIntegrator.cu:909-972):
//       c_new = (M_L (c/dt + M) - M K c~) / (M_L/dt + M sum V w FP),
//     or, in the implicit mode, the initial vectors of that solve (pcg.cu),
//   * velocity conditions (generalised PullGrid_kernal, TimeIntegrator.cu:169-261)
//     and the sticky walls of collideWithGround (TimeIntegrator.cu:117-165).
// Writes v (3), dc = c_new - c (update_grid_phase, ExplicitTimeIntegrator.cu:632-642)
// and c_new for G2P.
#include <cstdint>

#include "kernels.h"
#include "launch.cuh"

namespace gmpm {

constexpr int kGridThreads = 256;  // 4 grid pages per CTA

template <typename R>
__device__ __forceinline__ void grid_body(VB vb, const SceneDev<R>* __restrict__ sc, const BinDev& bin,
                                          const R* __restrict__ tile, R* __restrict__ nodes,
                                          double* __restrict__ diag, const PcgDev& pcg, Counters* cnt) {
    const int ng = min(cnt->n_grid_blocks, bin.ng_cap);
    const int node = threadIdx.x & 63;
    const int ci = node >> 4, cj = (node >> 2) & 3, ck = node & 3;
    const R dt = sc->dt, dx = sc->dx;
    const R Mob = sc->mobility;
    const double t_now = cnt->time;
    double dm = 0, dp0 = 0, dp1 = 0, dp2 = 0;
    for (int g = vb.b * 4 + (threadIdx.x >> 6); g < ng; g += vb.g * 4) {
        // fixed-order, compensated sum of the page tiles overlapping the node
        R ch[kP2GChannels], comp[kP2GChannels];
#pragma unroll
        for (int q = 0; q < kP2GChannels; ++q) ch[q] = comp[q] = R(0);
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            const int a = 4 * (d >> 2) + ci, b = 4 * ((d >> 1) & 1) + cj, c = 4 * (d & 1) + ck;
            if (a >= 6 || b >= 6 || c >= 6) continue;
            const int s = bin.grid_src[g * 8 + d];
            if (s < 0) continue;
            const R* T = tile + (int64_t)s * kP2GChannels * kWindowNodes + a * 36 + b * 6 + c;
#pragma unroll
            for (int q = 0; q < kP2GChannels; ++q) kahan_add(ch[q], comp[q], T[q * kWindowNodes]);
        }
        R out[kGridChannels] = {R(0), R(0), R(0), R(0), R(0)};
        const R mass = ch[CH_M];
        if (mass > R(0)) {
            dm += (double)mass;
            dp0 += (double)ch[CH_P0];
            dp1 += (double)ch[CH_P1];
            dp2 += (double)ch[CH_P2];
            const R cgrid = ch[CH_CW] / ch[CH_W];
            const R im = R(1) / mass;
            R v[3] = {ch[CH_P0] * im + sc->gravity[0] * dt, ch[CH_P1] * im + sc->gravity[1] * dt,
                      ch[CH_P2] * im + sc->gravity[2] * dt};
            R cnew = cgrid;
            if (sc->phase_field == GMPM_PHASE_FIELD_IMPLICIT) {
                // the solve's vectors (ExplicitTimeIntegrator.cu:913-935): rhs sum_p V w (c/dt + M)
                // (volP2G_APIC) as r with x0 = 0, Jacobi diagonal sum_p V w (FP M + 1/dt)
                // (preConditionP2G_APIC), mr = r / diag (precondition_subd), s = mr
                const PcgDev& P = pcg;
                const int64_t i = (int64_t)g * 64 + node;
                const double Md = (double)Mob, dtd = (double)dt;
                const double cg = (double)cgrid;
                const double dg = Md * (double)ch[CH_VWFP] + (double)ch[CH_VW] / dtd;
                const double b = (double)ch[CH_VW] * (cg / dtd + Md);
                const double mr = fabs(dg) >= 1e-30 ? b / dg : 0.0;
                P.x[i] = 0.0;
                P.r[i] = b;
                P.mr[i] = mr;
                P.s[i] = mr;
                P.q[i] = 0.0;
                P.d[i] = dg;
                P.cg[i] = cg;
                P.tag[i] = 1;
            } else if (sc->phase_field == GMPM_PHASE_FIELD_EXPLICIT) {
                const R diagv = ch[CH_VW] / dt + Mob * ch[CH_VWFP];
                const R rhs = ch[CH_VW] * (cgrid / dt + Mob) - Mob * ch[CH_KC];
                if (diagv != R(0)) cnew = rhs / diagv;
            }
            int gx, gy, gz;
            page_coords(bin.grid_keys[g], gx, gy, gz);
            const int idx[3] = {4 * gx + ci, 4 * gy + cj, 4 * gz + ck};
            const R pos[3] = {R(idx[0]) * dx, R(idx[1]) * dx, R(idx[2]) * dx};
            const VelocityConditions<R>& bc = sc->bc;
            for (int s = 0; s < bc.n_slabs; ++s) {
                const int ax = bc.slab_axis[s];
                if (pos[ax] >= bc.slab_lo[s] && pos[ax] <= bc.slab_hi[s]) {
                    v[0] = bc.slab_vel[s][0];
                    v[1] = bc.slab_vel[s][1];
                    v[2] = bc.slab_vel[s][2];
                }
            }
            for (int s = 0; s < bc.n_spheres; ++s) {
                R d2 = R(0);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const R dd = pos[a] - (bc.sph_c[s][a] + bc.sph_v[s][a] * R(t_now));
                    d2 += dd * dd;
                }
                if (d2 < bc.sph_r[s] * bc.sph_r[s]) {
                    v[0] = bc.sph_v[s][0];
                    v[1] = bc.sph_v[s][1];
                    v[2] = bc.sph_v[s][2];
                }
            }
            if (sc->wall_bc) {
                const int L = sc->wall_layers;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    if (idx[a] <= L && v[a] < R(0)) v[0] = v[1] = v[2] = R(0);
                    if (idx[a] > sc->res[a] - L && v[a] > R(0)) v[0] = v[1] = v[2] = R(0);
                }
            }
            out[GC_V0] = v[0];
            out[GC_V1] = v[1];
            out[GC_V2] = v[2];
            out[GC_DC] = cnew - cgrid;
            out[GC_CN] = cnew;
        }
        if (sc->phase_field == GMPM_PHASE_FIELD_IMPLICIT && !(mass > R(0))) {
            const int64_t i = (int64_t)g * 64 + node;
            pcg.x[i] = pcg.r[i] = pcg.mr[i] = pcg.s[i] = pcg.q[i] = pcg.d[i] = pcg.cg[i] = 0.0;
            pcg.tag[i] = 0;
        }
        R* N = nodes + (int64_t)g * kGridChannels * 64 + node;
#pragma unroll
        for (int q = 0; q < kGridChannels; ++q) N[q * 64] = out[q];
    }
    // FP64 conservation diagnostics of the P2G result
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dm += __shfl_down_sync(0xffffffffu, dm, o);
        dp0 += __shfl_down_sync(0xffffffffu, dp0, o);
        dp1 += __shfl_down_sync(0xffffffffu, dp1, o);
        dp2 += __shfl_down_sync(0xffffffffu, dp2, o);
    }
    if ((threadIdx.x & 31) == 0 && dm != 0.0) {
        atomicAdd(&diag[0], dm);
        atomicAdd(&diag[1], dp0);
        atomicAdd(&diag[2], dp1);
        atomicAdd(&diag[3], dp2);
    }
}

template <typename R>
__global__ void __launch_bounds__(kGridThreads)
    k_grid(const SceneDev<R>* __restrict__ sc, BinDev bin, const R* __restrict__ tile, R* __restrict__ nodes,
           double* __restrict__ diag, PcgDev pcg, Counters* cnt) {
    grid_body<R>(own_blocks(), sc, bin, tile, nodes, diag, pcg, cnt);
}

template <typename R>
__global__ void __launch_bounds__(kGridThreads)
    k_batch_grid(const SceneArgs<R>* __restrict__ A, const int32_t* __restrict__ start, int ns) {
    __shared__ SceneArgs<R> sa;
    VB vb;
    const SceneArgs<R>& a = batch_scene_args(A, start, ns, vb, sa);
    grid_body<R>(vb, a.sc, a.bin, reinterpret_cast<const R*>(a.grid.tile), reinterpret_cast<R*>(a.grid.nodes),
                 a.grid.diag, a.grid.pcg, a.cnt);
}

// One CTA per scene: clear the grid diagnostics the grid stage accumulates.
template <typename R>
__global__ void k_batch_zero_diag(const SceneArgs<R>* __restrict__ A, const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    if (threadIdx.x < 4) a.grid.diag[threadIdx.x] = 0.0;
}

template <typename R>
cudaError_t launch_batch_grid(const SceneArgs<R>* A, const BatchPlan& P, cudaStream_t s) {
    cudaError_t e = launch_kernel(k_batch_zero_diag<R>, dim3((unsigned)P.total[BM_ONE]), dim3(32), 0, s, A,
                                  P.start[BM_ONE], P.n_scenes);
    if (e == cudaSuccess)
        e = launch_kernel(k_batch_grid<R>, dim3((unsigned)P.total[BM_GRID]), dim3(kGridThreads), 0, s, A,
                          P.start[BM_GRID], P.n_scenes);
    return e;
}
template cudaError_t launch_batch_grid<float>(const SceneArgs<float>*, const BatchPlan&, cudaStream_t);
template cudaError_t launch_batch_grid<double>(const SceneArgs<double>*, const BatchPlan&, cudaStream_t);

template <typename R>
cudaError_t launch_grid(const SceneDev<R>* sc, BinDev bin, GridDev grid, Counters* cnt, LaunchCfg cfg,
                        cudaStream_t stream) {
    cudaMemsetAsync(grid.diag, 0, 4 * sizeof(double), stream);
    const int ctas = max(1, min(bin.ng_cap / 4 + 1, cfg.num_sms * 8));
    k_grid<R><<<ctas, kGridThreads, 0, stream>>>(sc, bin, reinterpret_cast<const R*>(grid.tile),
                                                 reinterpret_cast<R*>(grid.nodes), grid.diag, grid.pcg, cnt);
    return cudaGetLastError();
}

template cudaError_t launch_grid<float>(const SceneDev<float>*, BinDev, GridDev, Counters*, LaunchCfg, cudaStream_t);
template cudaError_t launch_grid<double>(const SceneDev<double>*, BinDev, GridDev, Counters*, LaunchCfg,
                                         cudaStream_t);

}  // namespace gmpm
