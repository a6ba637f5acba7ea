// Scene initialisation (first constitutive evaluation), FP64 particle
// diagnostics and field readback.
#include <cstdint>

#include "constitutive.cuh"
#include "kernels.h"

namespace gmpm {

// The reference's first applyVonMises (or its other energy models' contribution
// kernels) runs at the start of substep 1 with the
// initial state g = 1 (initArray, Particle_kernal.cu:451-454); here it runs at
// scene creation so every substep can start at P2G.
template <typename R>
__global__ void k_init_stress(const SceneDev<R>* __restrict__ sc, PState<R> st, PAux<R> aux, int64_t n,
                              Counters* cnt) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    R F[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = st.F(q, p);
    const int mat = (int)(st.id[p] >> 28);
    StressOut<R> so;
    constitutive_update<R, R>(sc->mat[mat], sc->V0, sc->dx, F, R(1), st.alpha(p), st.c[p], st.psi(p), so);
    if (!so.svd_ok) raise_flag(cnt, GMPM_FLAG_SVD_NOCONVERGE);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        st.F(q, p) = so.F[q];
        aux.B[q][p] = R(0);
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) aux.sigma[q][p] = so.sigma[q];
#pragma unroll
    for (int a = 0; a < 3; ++a) aux.q[a][p] = R(0);
    st.alpha(p) = so.alpha;
    st.psi(p) = so.psi;
    aux.vol[p] = so.vol;
    aux.FP[p] = so.FP;
}

template <typename R>
cudaError_t launch_init_stress(const SceneDev<R>* sc, const PState<R>& st, const PAux<R>& aux, int64_t n,
                               Counters* cnt, cudaStream_t stream) {
    const int T = 128;
    k_init_stress<R><<<(unsigned)((n + T - 1) / T), T, 0, stream>>>(sc, st, aux, n, cnt);
    return cudaGetLastError();
}
template cudaError_t launch_init_stress<float>(const SceneDev<float>*, const PState<float>&, const PAux<float>&,
                                               int64_t, Counters*, cudaStream_t);
template cudaError_t launch_init_stress<double>(const SceneDev<double>*, const PState<double>&,
                                                const PAux<double>&, int64_t, Counters*, cudaStream_t);

// ---------------------------------------------------------------------------

template <typename R>
__global__ void k_particle_diag(PState<R> st, PAux<R> aux, int64_t n, double* acc) {
    double m = 0, p0 = 0, p1 = 0, p2 = 0, ke = 0, vmax = 0, cmin = 1e300;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (int64_t)gridDim.x * blockDim.x) {
        const double mm = st.m[p];
        const double v0 = aux.v[0][p], v1 = aux.v[1][p], v2 = aux.v[2][p];
        m += mm;
        p0 += mm * v0;
        p1 += mm * v1;
        p2 += mm * v2;
        const double v2s = v0 * v0 + v1 * v1 + v2 * v2;
        ke += 0.5 * mm * v2s;
        vmax = fmax(vmax, sqrt(v2s));
        cmin = fmin(cmin, (double)st.c[p]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_down_sync(0xffffffffu, m, o);
        p0 += __shfl_down_sync(0xffffffffu, p0, o);
        p1 += __shfl_down_sync(0xffffffffu, p1, o);
        p2 += __shfl_down_sync(0xffffffffu, p2, o);
        ke += __shfl_down_sync(0xffffffffu, ke, o);
        vmax = fmax(vmax, __shfl_down_sync(0xffffffffu, vmax, o));
        cmin = fmin(cmin, __shfl_down_sync(0xffffffffu, cmin, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], m);
        atomicAdd(&acc[1], p0);
        atomicAdd(&acc[2], p1);
        atomicAdd(&acc[3], p2);
        atomicAdd(&acc[4], ke);
        // non-negative doubles order like their bit patterns
        atomicMax(reinterpret_cast<unsigned long long*>(&acc[5]), (unsigned long long)__double_as_longlong(vmax));
        if (cmin >= 0.0)
            atomicMin(reinterpret_cast<unsigned long long*>(&acc[6]), (unsigned long long)__double_as_longlong(cmin));
    }
}

__global__ void k_diag_init(double* acc) {
    for (int q = 0; q < 8; ++q) acc[q] = 0.0;
    acc[6] = 1e300;
}

template <typename R>
cudaError_t launch_particle_diag(const PState<R>& st, const PAux<R>& aux, int64_t n, double* acc,
                                 cudaStream_t stream) {
    k_diag_init<<<1, 1, 0, stream>>>(acc);
    const int T = 256;
    const int64_t blocks = (n + T - 1) / T;
    k_particle_diag<R><<<(unsigned)(blocks < 1184 ? blocks : 1184), T, 0, stream>>>(st, aux, n, acc);
    return cudaGetLastError();
}
template cudaError_t launch_particle_diag<float>(const PState<float>&, const PAux<float>&, int64_t, double*,
                                                 cudaStream_t);
template cudaError_t launch_particle_diag<double>(const PState<double>&, const PAux<double>&, int64_t, double*,
                                                  cudaStream_t);

// ---------------------------------------------------------------------------

struct FieldPlanes {
    const void* plane[9];
    int step[9];  // elements between particles: 1 for a plane, 4 for a component of a four-wide word
    int comps;
    int is_id;
};

template <typename R>
__host__ FieldPlanes field_planes(const PState<R>& st, const PAux<R>& aux, int field) {
    FieldPlanes f{};
    for (int q = 0; q < 9; ++q) f.step[q] = 1;
    auto set = [&](int nc, auto* const* planes) {
        f.comps = nc;
        for (int q = 0; q < nc; ++q) f.plane[q] = planes[q];
    };
    auto word_component = [&](int slot, int q) {  // F(q) for q < 9; alpha and psi_max follow F8
        f.plane[slot] = reinterpret_cast<const R*>(st.fw[q >> 2]) + (q & 3);
        f.step[slot] = 4;
    };
    switch (field) {
        case GMPM_FIELD_POSITION: set(3, st.x); break;
        case GMPM_FIELD_VELOCITY: set(3, aux.v); break;
        case GMPM_FIELD_F:
            f.comps = 9;
            for (int q = 0; q < 9; ++q) word_component(q, q);
            break;
        case GMPM_FIELD_B: set(9, aux.B); break;
        case GMPM_FIELD_DAMAGE: f.comps = 1; f.plane[0] = st.c; break;
        case GMPM_FIELD_ALPHA: f.comps = 1; word_component(0, 9); break;
        case GMPM_FIELD_PSI_MAX: f.comps = 1; word_component(0, 10); break;
        case GMPM_FIELD_STRESS: set(6, aux.sigma); break;
        case GMPM_FIELD_VOLUME: f.comps = 1; f.plane[0] = aux.vol; break;
        case GMPM_FIELD_FP: f.comps = 1; f.plane[0] = aux.FP; break;
        case GMPM_FIELD_PF_FLUX: set(3, aux.q); break;
        case GMPM_FIELD_MASS: f.comps = 1; f.plane[0] = st.m; break;
        case GMPM_FIELD_ID: f.comps = 1; f.plane[0] = st.id; f.is_id = 1; break;
        default: f.comps = 0; break;
    }
    return f;
}

template <typename R>
__global__ void k_pack_field(FieldPlanes f, const uint32_t* __restrict__ ids, int dtype, int order, int64_t n,
                             void* out) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int64_t dst = (order == GMPM_ORDER_ORIGINAL) ? (int64_t)(ids[p] & 0x0fffffffu) : p;
    if (dst >= n) return;
    for (int q = 0; q < f.comps; ++q) {
        double v;
        if (f.is_id)
            v = (double)(reinterpret_cast<const uint32_t*>(f.plane[q])[p] & 0x0fffffffu);
        else
            v = (double)reinterpret_cast<const R*>(f.plane[q])[p * f.step[q]];
        const int64_t e = dst * f.comps + q;
        if (dtype == GMPM_DTYPE_F64)
            reinterpret_cast<double*>(out)[e] = v;
        else if (dtype == GMPM_DTYPE_F32)
            reinterpret_cast<float*>(out)[e] = (float)v;
        else
            reinterpret_cast<int32_t*>(out)[e] = (int32_t)v;
    }
}

int field_components(int field) {
    switch (field) {
        case GMPM_FIELD_POSITION: case GMPM_FIELD_VELOCITY: case GMPM_FIELD_PF_FLUX: return 3;
        case GMPM_FIELD_F: case GMPM_FIELD_B: return 9;
        case GMPM_FIELD_STRESS: return 6;
        case GMPM_FIELD_DAMAGE: case GMPM_FIELD_ALPHA: case GMPM_FIELD_PSI_MAX: case GMPM_FIELD_VOLUME:
        case GMPM_FIELD_FP: case GMPM_FIELD_MASS: case GMPM_FIELD_ID: return 1;
        default: return 0;
    }
}

template <typename R>
cudaError_t launch_pack_field(const PState<R>& st, const PAux<R>& aux, int field, int dtype, int order, int64_t n,
                              void* out, cudaStream_t stream) {
    FieldPlanes f = field_planes(st, aux, field);
    const int T = 256;
    k_pack_field<R><<<(unsigned)((n + T - 1) / T), T, 0, stream>>>(f, st.id, dtype, order, n, out);
    return cudaGetLastError();
}
template cudaError_t launch_pack_field<float>(const PState<float>&, const PAux<float>&, int, int, int, int64_t,
                                              void*, cudaStream_t);
template cudaError_t launch_pack_field<double>(const PState<double>&, const PAux<double>&, int, int, int, int64_t,
                                               void*, cudaStream_t);

}  // namespace gmpm
