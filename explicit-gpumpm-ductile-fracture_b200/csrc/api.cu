// C-ABI of the substep library (include/gmpm.h): context and scene lifetime,
// stepping, readback and diagnostics.  Every entry point returns a status;
// no call exits the process.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <atomic>

#include "kernels.h"
#include "scene.h"

namespace gmpm {

gmpm_status flags_status(unsigned int f) {
    if (f & GMPM_FLAG_COPY_TIMEOUT) return GMPM_CUDA_ERROR;
    if (f & GMPM_FLAG_TABLE_OVERFLOW) return GMPM_TABLE_OVERFLOW;
    if (f & GMPM_FLAG_OUT_OF_DOMAIN) return GMPM_OUT_OF_DOMAIN;
    if (f & GMPM_FLAG_NONFINITE) return GMPM_NONFINITE;
    return GMPM_OK;
}

gmpm_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return GMPM_OK;
    if (e == cudaErrorMemoryAllocation) return GMPM_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return GMPM_NO_DEVICE;
    return GMPM_CUDA_ERROR;
}

std::atomic<uint64_t> g_scene_uid{1};

// Checkpoint file: this header, the scene description, then every particle
// plane of the state (n values each, in the internal order).
constexpr char kSnapshotMagic[8] = {'G', 'M', 'P', 'M', 'S', 'N', 'A', 'P'};
constexpr uint32_t kSnapshotVersion = 2;  // 2: F and the plastic state as four-wide words
struct SnapshotHeader {
    char magic[8];
    uint32_t version;
    uint32_t real_bytes;
    uint32_t desc_bytes;
    uint32_t _pad;
    int64_t n;
    double time;
    int64_t substeps;
    double dt;
};

namespace {

#define GMPM_TRY(expr)                                   \
    do {                                                 \
        cudaError_t e_ = (expr);                         \
        if (e_ != cudaSuccess) return cuda_status(e_);   \
    } while (0)

// Gauss-Jordan with the full pivot search of the reference's Inverse()
// (ExplicitTimeIntegrator.cu:71-129); evaluated once per material on the host.
void stiffness_inverse(double lambda, double mu, double* D) {
    double mat[9] = {2 * mu + lambda, lambda, lambda, lambda, 2 * mu + lambda, lambda, lambda, lambda, 2 * mu + lambda};
    int swapR[3], swapC[3];
    int pivot[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        int pr = 0, pc = 0;
        double maxv = 0;
        for (int j = 0; j < 3; ++j)
            if (pivot[j] != 1)
                for (int k = 0; k < 3; ++k)
                    if (pivot[k] == 0 && mat[j * 3 + k] > maxv) {
                        maxv = mat[j * 3 + k];
                        pr = j;
                        pc = k;
                    }
        if (pr != pc)
            for (int j = 0; j < 3; ++j) {
                const double t = mat[pr * 3 + j];
                mat[pr * 3 + j] = mat[pc * 3 + j];
                mat[pc * 3 + j] = t;
            }
        swapC[i] = pc;
        swapR[i] = pr;
        ++pivot[i];
        const double inv = 1.0 / mat[pc * 3 + pc];
        mat[pc * 3 + pc] = 1;
        for (int j = 0; j < 3; ++j) mat[pc * 3 + j] *= inv;
        for (int j = 0; j < 3; ++j)
            if (j != pc) {
                const double ratio = mat[j * 3 + pc];
                mat[j * 3 + pc] = 0.0;
                for (int k = 0; k < 3; ++k) mat[j * 3 + k] -= mat[pc * 3 + k] * ratio;
            }
    }
    for (int i = 0; i < 3; ++i)
        if (swapR[i] != swapC[i])
            for (int j = 0; j < 3; ++j) {
                const double t = mat[j * 3 + swapC[i]];
                mat[j * 3 + swapC[i]] = mat[j * 3 + swapR[i]];
                mat[j * 3 + swapR[i]] = t;
            }
    for (int q = 0; q < 9; ++q) D[q] = mat[q];
}

template <typename R>
void fill_velocity_conditions(const gmpm_slab_bc* slabs, int n_slabs, const gmpm_sphere_bc* spheres, int n_spheres,
                              VelocityConditions<R>& bc) {
    std::memset(&bc, 0, sizeof(bc));
    bc.n_slabs = n_slabs;
    bc.n_spheres = n_spheres;
    for (int q = 0; q < n_slabs; ++q) {
        bc.slab_axis[q] = slabs[q].axis;
        bc.slab_lo[q] = (R)slabs[q].lo;
        bc.slab_hi[q] = (R)slabs[q].hi;
        for (int a = 0; a < 3; ++a) bc.slab_vel[q][a] = (R)slabs[q].velocity[a];
    }
    for (int q = 0; q < n_spheres; ++q) {
        for (int a = 0; a < 3; ++a) {
            bc.sph_c[q][a] = (R)spheres[q].center[a];
            bc.sph_v[q][a] = (R)spheres[q].velocity[a];
        }
        bc.sph_r[q] = (R)spheres[q].radius;
    }
}

template <typename R>
void fill_scene_dev(const gmpm_scene_desc& d, int key_bits, SceneDev<R>& s) {
    std::memset(&s, 0, sizeof(s));
    s.dx = (R)d.dx;
    s.inv_dx = (R)(1.0 / d.dx);
    s.dt = (R)d.dt;
    s.Dinv = (R)(4.0 / (d.dx * d.dx));
    for (int a = 0; a < 3; ++a) {
        s.gravity[a] = (R)d.gravity[a];
        s.res[a] = d.grid_res[a];
    }
    s.V0 = (R)d.particle_volume;
    s.key_bits = key_bits;
    s.n_materials = d.n_materials;
    for (int m = 0; m < d.n_materials; ++m) {
        const gmpm_material& in = d.materials[m];
        MaterialDev<R>& o = s.mat[m];
        // Lame parameters as ElasticMaterial (Materials.cpp:4-13)
        const double E = in.youngs_modulus, nu = in.poisson_ratio;
        const double lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
        const double mu = E / (2 * (1 + nu));
        const double kappa = E / (3 * (1 - 2 * nu));
        double D[9];
        stiffness_inverse(lambda, mu, D);
        o.lambda = (R)lambda;
        o.mu = (R)mu;
        o.kappa = (R)kappa;
        for (int q = 0; q < 9; ++q) o.D[q] = (R)D[q];
        o.yield_stress = (R)in.yield_stress;
        o.hardening = (R)in.hardening;
        o.hardening_law = in.hardening_law;
        o.energy_model = in.energy_model;
        o.alpha_cap = (R)in.alpha_cap;
        o.dlambda_cap = (R)in.dlambda_cap;
        o.strain_cap = (R)in.strain_cap;
        o.psi_cap = (R)in.psi_cap;
        o.fracture_energy = (R)in.fracture_energy;
        o.softening_onset = (R)in.softening_onset;
        o.residual_fracture = (R)in.residual_fracture;
        o.theta = (R)(float)in.theta;
        o.one_minus_theta = (R)(1.0f - (float)in.theta);
        o.length_scale = (R)in.length_scale;
        o.mobility = (R)in.mobility;
    }
    s.mobility = (R)d.materials[0].mobility;
    s.wall_bc = d.wall_bc;
    s.wall_layers = d.wall_layers;
    fill_velocity_conditions<R>(d.slabs, d.n_slab_bcs, d.spheres, d.n_sphere_bcs, s.bc);
    s.phase_field = d.phase_field;
    s.fp64_svd_fallback = (d.precision == GMPM_PRECISION_FP32_FP64SVD);
    s.svd_fallback_ratio = (R)d.svd_fallback_ratio;
    s.dx_d = d.dx;
    s.inv_dx_d = 1.0 / d.dx;
    s.adaptive_dt = d.adaptive_dt;
    s.pcg_max_combine = d.pcg_max_combine;
    s.pcg_tolerance = d.pcg_tolerance;
    s.dt_max = d.dt;
    s.cfl_dx = d.dx * (d.cfl_number > 0 ? d.cfl_number : (double)0.3f);
}

// First substep's dt in adaptive mode: the CFL bound of the initial velocities
// (MPMSimulator::computeDt, Simulator.cpp:200-225).
double initial_cfl_dt(const gmpm_scene_desc& d, const gmpm_particle_init& init) {
    double v2max = 0.0;
    if (init.velocities)
        for (int64_t p = 0; p < init.count; ++p) {
            const double* v = init.velocities + 3 * p;
            v2max = std::max(v2max, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        }
    const double vmax = std::sqrt(v2max);
    const double cdx = d.dx * (d.cfl_number > 0 ? d.cfl_number : (double)0.3f);
    return (vmax > 0 && cdx / vmax < d.dt) ? cdx / vmax : d.dt;
}

gmpm_status validate(const gmpm_scene_desc* d, const gmpm_particle_init* init) {
    if (!d || !init || !init->positions || !init->masses) return GMPM_INVALID_ARG;
    if (init->count <= 0 || init->count >= (int64_t(1) << 28)) return GMPM_INVALID_ARG;
    if (!(d->dx > 0) || !(d->dt > 0) || !(d->particle_volume > 0)) return GMPM_INVALID_ARG;
    for (int a = 0; a < 3; ++a)
        if (d->grid_res[a] < 8 || d->grid_res[a] > 1019) return GMPM_INVALID_ARG;
    if (d->n_materials < 1 || d->n_materials > GMPM_MAX_MATERIALS) return GMPM_INVALID_ARG;
    for (int m = 0; m < d->n_materials; ++m) {
        const gmpm_material& mt = d->materials[m];
        if (!(mt.youngs_modulus > 0) || !(mt.poisson_ratio >= 0) || !(mt.poisson_ratio < 0.5)) return GMPM_INVALID_ARG;
        if (!(mt.fracture_energy > 0)) return GMPM_INVALID_ARG;
        if (mt.hardening_law != GMPM_HARDENING_EXPONENTIAL && mt.hardening_law != GMPM_HARDENING_LINEAR)
            return GMPM_INVALID_ARG;
        if (mt.energy_model < GMPM_ENERGY_VON_MISES_FRACTURE || mt.energy_model > GMPM_ENERGY_NEO_HOOKEAN_FRACTURE)
            return GMPM_INVALID_ARG;
    }
    if (d->n_slab_bcs < 0 || d->n_slab_bcs > GMPM_MAX_SLAB_BCS) return GMPM_INVALID_ARG;
    if (d->n_sphere_bcs < 0 || d->n_sphere_bcs > GMPM_MAX_SPHERE_BCS) return GMPM_INVALID_ARG;
    for (int q = 0; q < d->n_slab_bcs; ++q)
        if (d->slabs[q].axis < 0 || d->slabs[q].axis > 2) return GMPM_INVALID_ARG;
    if (d->precision < 0 || d->precision > 2) return GMPM_INVALID_ARG;
    if (d->phase_field < 0 || d->phase_field > 2) return GMPM_INVALID_ARG;
    if (d->phase_field == GMPM_PHASE_FIELD_IMPLICIT &&
        (d->pcg_max_iterations < 1 || d->pcg_max_iterations > 10000 || !(d->pcg_tolerance >= 0)))
        return GMPM_INVALID_ARG;
    if (d->block_capacity < 0) return GMPM_INVALID_ARG;
    if (d->adaptive_dt < 0 || d->adaptive_dt > 1 || !(d->cfl_number >= 0)) return GMPM_INVALID_ARG;
    if (init->material_ids)
        for (int64_t p = 0; p < init->count; ++p)
            if (init->material_ids[p] < 0 || init->material_ids[p] >= d->n_materials) return GMPM_INVALID_ARG;
    return GMPM_OK;
}

int bit_width(unsigned v) {
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

inline size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace

template <typename R>
struct Scene : SceneBase {
    gmpm_context* ctx = nullptr;
    gmpm_scene_desc desc{};
    int64_t n = 0;
    int64_t stride = 0;  // plane stride (elements)
    SceneDev<R>* d_sc = nullptr;
    SceneDev<double>* d_sc64 = nullptr;
    void* pstore = nullptr;
    PState<R> st[2];
    PAux<R> aux;
    int cur = 0;
    BinDev bin{};
    ScanScratch scan{};
    GridDev grid{};
    Counters* d_cnt = nullptr;
    double* d_pdiag = nullptr;  // [8]
    void* staging = nullptr;
    size_t staging_bytes = 0;
    std::vector<void*> allocs;
    bool binned = false;  // binning of the current positions is valid
    // bin.keys and bin.page_flag hold the keys and pages of the current
    // positions (set by a key pass or by the G2P that wrote them), so the next
    // binning skips its key pass
    bool keys_fresh = false;
    int64_t launches = 0;  // kernels launched by this scene
    uint64_t uid_ = g_scene_uid++;
    int share_ = 0;        // SMs the launch shapes are sized for (0: all)
    size_t dev_bytes_ = 0;

    // Device memory comes from the device's stream-ordered pool.  A scene
    // released on a stream (the serving loop, after its last use there) frees
    // it on that stream without synchronising the device; otherwise the
    // device is synchronised first, since the scene's work may be in flight
    // on any stream.
    cudaStream_t release_stream_ = nullptr;
    bool release_on_stream_ = false;
    void set_release_stream(cudaStream_t s) override {
        release_stream_ = s;
        release_on_stream_ = true;
    }

    ~Scene() override {
        cudaStream_t rs = release_stream_;
        if (!release_on_stream_) {
            cudaDeviceSynchronize();
            rs = 0;
        }
        for (void* p : allocs) cudaFreeAsync(p, rs);
        if (staging) cudaFreeAsync(staging, rs);
        if (copy_stream_) cudaStreamSynchronize(copy_stream_);
        for (int b = 0; b < 2; ++b) {
            if (rstage_[b]) cudaFreeAsync(rstage_[b], rs);
            if (rstage_packed_[b]) cudaEventDestroy(rstage_packed_[b]);
            if (rstage_free_[b]) cudaEventDestroy(rstage_free_[b]);
        }
        if (copy_stream_) cudaStreamDestroy(copy_stream_);
        if (pcg_done_host) cudaFreeHost(pcg_done_host);
        if (bc_staging) cudaFreeHost(bc_staging);
        if (dt_staging) cudaFreeHost(dt_staging);
        for (cudaEvent_t e : dt_done)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : bc_done)
            if (e) cudaEventDestroy(e);
    }

    template <typename T>
    cudaError_t alloc(T** p, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, count * sizeof(T) + 16, 0);
        if (e != cudaSuccess) return e;
        allocs.push_back(q);
        dev_bytes_ += count * sizeof(T) + 16;
        *p = reinterpret_cast<T*>(q);
        return cudaSuccess;
    }

    LaunchCfg cfg() const {
        int other = 0;
        for (int m = 0; m < desc.n_materials; ++m) other |= desc.materials[m].energy_model != GMPM_ENERGY_VON_MISES_FRACTURE;
        return LaunchCfg{share_ > 0 ? std::min(share_, ctx->num_sms) : ctx->num_sms, desc.deterministic,
                         desc.pcg_max_combine, desc.materials[0].mobility, desc.pcg_tolerance, other};
    }
    bool implicit_pf() const { return desc.phase_field == GMPM_PHASE_FIELD_IMPLICIT; }
    int* pcg_done_host = nullptr;  // pinned: the solve's done flag, read between iterations

    gmpm_status create(gmpm_context* c, const gmpm_scene_desc* d, const gmpm_particle_init* init) {
        ctx = c;
        desc = *d;
        n = init->count;
        // Planes are padded so that a bulk copy of a window of previous slots
        // around any chunk stays inside the allocation.
        stride = (int64_t)round_up((size_t)n, 64) + kPlanePad;
        GMPM_TRY(cudaSetDevice(ctx->device));
        // key space of the grid (page coordinates incl. the + neighbour page)
        int maxb = 0;
        for (int a = 0; a < 3; ++a) maxb = std::max(maxb, (d->grid_res[a] - 3) >> 2);
        const int key_bits = bit_width((unsigned)(maxb + 1));
        if (3 * key_bits + 6 > 32) return GMPM_INVALID_ARG;
        const uint32_t key_space = 1u << (3 * key_bits);

        SceneDev<R> h{};
        fill_scene_dev<R>(desc, key_bits, h);
        SceneDev<double> h64{};
        fill_scene_dev<double>(desc, key_bits, h64);
        if (desc.adaptive_dt) {
            const double dt0 = initial_cfl_dt(desc, *init);
            h.dt = (R)dt0;
            h64.dt = dt0;
        }
        GMPM_TRY(alloc(&d_sc, 1));
        GMPM_TRY(alloc(&d_sc64, 1));
        GMPM_TRY(cudaMemcpy(d_sc, &h, sizeof(h), cudaMemcpyHostToDevice));
        GMPM_TRY(cudaMemcpy(d_sc64, &h64, sizeof(h64), cudaMemcpyHostToDevice));
        GMPM_TRY(alloc(&d_cnt, 1));
        GMPM_TRY(cudaMemset(d_cnt, 0, sizeof(Counters)));
        GMPM_TRY(alloc(&d_pdiag, 8));
        GMPM_TRY(alloc(&grid.diag, 8));
        GMPM_TRY(cudaMemset(grid.diag, 0, 8 * sizeof(double)));

        // particle planes: 2 x (x3 c m + 3 four-wide words F/alpha/psi) + aux (v3 B9 sigma6 vol FP q3),
        // + 2 id planes
        const int state_planes = 5 + 3 * 4, aux_planes = 23;
        const size_t nplanes = 2 * state_planes + aux_planes;
        const size_t plane_bytes = round_up((size_t)stride * sizeof(R), 256);
        const size_t id_bytes = round_up((size_t)stride * sizeof(uint32_t), 256);
        GMPM_TRY(cudaMallocAsync(&pstore, nplanes * plane_bytes + 2 * id_bytes, 0));
        allocs.push_back(pstore);
        dev_bytes_ += nplanes * plane_bytes + 2 * id_bytes;
        char* base = reinterpret_cast<char*>(pstore);
        auto next = [&]() {
            R* p = reinterpret_cast<R*>(base);
            base += plane_bytes;
            return p;
        };
        auto next_word = [&]() {
            Word4<R>* p = reinterpret_cast<Word4<R>*>(base);
            base += 4 * plane_bytes;
            return p;
        };
        for (int b = 0; b < 2; ++b) {
            st[b].stride = stride;
            for (int a = 0; a < 3; ++a) st[b].x[a] = next();
            for (int k = 0; k < 3; ++k) st[b].fw[k] = next_word();
            st[b].c = next();
            st[b].m = next();
        }
        for (int a = 0; a < 3; ++a) aux.v[a] = next();
        for (int q = 0; q < 9; ++q) aux.B[q] = next();
        for (int q = 0; q < 6; ++q) aux.sigma[q] = next();
        aux.vol = next();
        aux.FP = next();
        for (int a = 0; a < 3; ++a) aux.q[a] = next();
        for (int b = 0; b < 2; ++b) {
            st[b].id = reinterpret_cast<uint32_t*>(base);
            base += id_bytes;
        }

        // upload the initial state into buffer 0 (original order)
        {
            std::vector<R> tmp((size_t)n);
            for (int a = 0; a < 3; ++a) {
                for (int64_t p = 0; p < n; ++p) tmp[p] = (R)init->positions[3 * p + a];
                GMPM_TRY(cudaMemcpy(st[0].x[a], tmp.data(), n * sizeof(R), cudaMemcpyHostToDevice));
                for (int64_t p = 0; p < n; ++p) tmp[p] = init->velocities ? (R)init->velocities[3 * p + a] : R(0);
                GMPM_TRY(cudaMemcpy(aux.v[a], tmp.data(), n * sizeof(R), cudaMemcpyHostToDevice));
            }
            for (int64_t p = 0; p < n; ++p) tmp[p] = (R)init->masses[p];
            GMPM_TRY(cudaMemcpy(st[0].m, tmp.data(), n * sizeof(R), cudaMemcpyHostToDevice));
            {
                // F = I (F0, F4 and F8 are the diagonal), alpha = psi_max = 0
                const Word4<R> w{{R(1), R(0), R(0), R(0)}};
                std::vector<Word4<R>> words((size_t)n, w);
                for (int k = 0; k < 3; ++k)
                    GMPM_TRY(cudaMemcpy(st[0].fw[k], words.data(), n * sizeof(Word4<R>), cudaMemcpyHostToDevice));
            }
            for (int64_t p = 0; p < n; ++p) tmp[p] = R(1);
            GMPM_TRY(cudaMemcpy(st[0].c, tmp.data(), n * sizeof(R), cudaMemcpyHostToDevice));
            std::vector<uint32_t> ids((size_t)n);
            for (int64_t p = 0; p < n; ++p)
                ids[p] = (uint32_t)p | ((uint32_t)(init->material_ids ? init->material_ids[p] : 0) << 28);
            GMPM_TRY(cudaMemcpy(st[0].id, ids.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice));
        }
        GMPM_TRY(launch_init_stress<R>(d_sc, st[0], aux, n, d_cnt, 0));

        // binning storage; page capacities from a first count on the device
        bin.n = n;
        bin.key_space = key_space;
        GMPM_TRY(alloc(&bin.keys, (size_t)n));
        GMPM_TRY(alloc(&bin.keys_sorted, (size_t)n));
        GMPM_TRY(alloc(&bin.perm, (size_t)n));
        GMPM_TRY(alloc(&bin.page_flag, key_space));
        GMPM_TRY(alloc(&bin.page_rank, key_space));
        GMPM_TRY(alloc(&bin.grid_flag, key_space));
        GMPM_TRY(alloc(&bin.grid_rank, key_space));
        int nb0 = 0, ng0 = 0;
        {
            // a provisional pass with tiny capacities only to count pages
            bin.nb_cap = 1;
            bin.ng_cap = 1;
            const int64_t scan_n = key_space;
            scan.capacity = scan_scratch_elems(scan_n);
            int32_t* ts = nullptr;
            GMPM_TRY(alloc(&ts, (size_t)scan.capacity));
            scan.tile_sums = ts;
            GMPM_TRY(count_pages(&nb0, &ng0));
        }
        int64_t nb_cap = desc.block_capacity > 0 ? desc.block_capacity : std::max<int64_t>(2 * (int64_t)nb0, nb0 + 256);
        int64_t ng_cap = std::max<int64_t>(2 * (int64_t)ng0, ng0 + 512);
        if (desc.block_capacity > 0) ng_cap = std::max<int64_t>(ng_cap, std::min<int64_t>(8 * nb_cap, key_space));
        nb_cap = std::min<int64_t>(nb_cap, key_space);
        ng_cap = std::min<int64_t>(ng_cap, key_space);
        if (nb_cap < nb0) return GMPM_TABLE_OVERFLOW;
        bin.nb_cap = (int32_t)nb_cap;
        bin.ng_cap = (int32_t)ng_cap;
        GMPM_TRY(alloc(&bin.block_keys, (size_t)nb_cap));
        GMPM_TRY(alloc(&bin.cell_count, (size_t)nb_cap * 64));
        GMPM_TRY(alloc(&bin.cell_start, (size_t)nb_cap * 64 + 1));
        GMPM_TRY(alloc(&bin.grid_keys, (size_t)ng_cap));
        GMPM_TRY(alloc(&bin.adj, (size_t)nb_cap * 8));
        GMPM_TRY(alloc(&bin.grid_src, (size_t)ng_cap * 8));
        {
            const int64_t scan_n = std::max<int64_t>(key_space, nb_cap * 64);
            scan.capacity = scan_scratch_elems(scan_n);
            int32_t* ts = nullptr;
            GMPM_TRY(alloc(&ts, (size_t)scan.capacity));
            scan.tile_sums = ts;
        }
        R* tile = nullptr;
        R* nodes = nullptr;
        GMPM_TRY(alloc(&tile, (size_t)nb_cap * kP2GChannels * kWindowNodes));
        GMPM_TRY(alloc(&nodes, (size_t)ng_cap * kGridChannels * 64));
        grid.tile = tile;
        grid.nodes = nodes;
        grid.pcg = PcgDev{};
        if (implicit_pf()) {
            const size_t nn = (size_t)ng_cap * 64;
            PcgDev& P = grid.pcg;
            for (double** v : {&P.x, &P.r, &P.mr, &P.s, &P.q, &P.d, &P.cg}) GMPM_TRY(alloc(v, nn));
            GMPM_TRY(alloc(&P.tag, nn));
            GMPM_TRY(alloc(&P.col, (size_t)3 * n));
            P.nparts_cap = (int64_t)(nn / 128 + 1);
            GMPM_TRY(alloc(&P.part, (size_t)3 * P.nparts_cap));
            GMPM_TRY(alloc(&P.scal, 1));
            GMPM_TRY(cudaMemset(P.scal, 0, sizeof(PcgScalars)));
            P.n = n;
            GMPM_TRY(cudaMallocHost(reinterpret_cast<void**>(&pcg_done_host), sizeof(int)));
        }
        GMPM_TRY(prepare_p2g<R>());
        GMPM_TRY(prepare_g2p<R>());
        GMPM_TRY(cudaMemset(d_cnt, 0, sizeof(Counters)));
        // keys of the initial positions into the cleared counters (an
        // out-of-domain particle raises its flag here)
        GMPM_TRY(refresh_keys(0));
        // creation work ran on the legacy stream; waiting for it alone leaves
        // other streams' work (e.g. a serving batch) running
        GMPM_TRY(cudaStreamSynchronize(0));
        return GMPM_OK;
    }

    // Count active and grid pages of the current positions (creation only).
    cudaError_t count_pages(int* nb, int* ng) {
        const int T = 256;
        const unsigned gk = (bin.key_space + T - 1) / T;
        cudaMemset(bin.page_flag, 0, bin.key_space);
        cudaMemset(bin.grid_flag, 0, bin.key_space);
        launch_keys_only(0);
        scan_exclusive<uint8_t>(bin.page_flag, bin.page_rank, (int64_t)bin.key_space, &d_cnt->n_blocks, scan, 0);
        mark_grid(0);
        scan_exclusive<uint8_t>(bin.grid_flag, bin.grid_rank, (int64_t)bin.key_space, &d_cnt->n_grid_blocks, scan, 0);
        (void)gk;
        Counters h{};
        cudaError_t e = cudaMemcpy(&h, d_cnt, sizeof(h), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return e;
        *nb = h.n_blocks;
        *ng = h.n_grid_blocks;
        return cudaGetLastError();
    }
    void launch_keys_only(cudaStream_t s);
    void mark_grid(cudaStream_t s);

    // A key pass over the current positions: keys and page flags.
    cudaError_t refresh_keys(cudaStream_t s) {
        cudaError_t e = cudaMemsetAsync(bin.page_flag, 0, bin.key_space, s);
        if (e == cudaSuccess) e = launch_keys<R>(d_sc, st[cur], bin, d_cnt, s);
        if (e == cudaSuccess) keys_fresh = true;
        return e;
    }
    gmpm_status ensure_keys(cudaStream_t s) override {
        if (keys_fresh) return GMPM_OK;
        GMPM_TRY(cudaSetDevice(ctx->device));
        launches += 1;
        GMPM_TRY(refresh_keys(s));
        return GMPM_OK;
    }

    gmpm_status do_bin(cudaStream_t s) {
        GMPM_TRY(launch_binning<R>(d_sc, st[cur], bin, scan, d_cnt, cfg().num_sms, s));
        binned = true;
        keys_fresh = true;
        return GMPM_OK;
    }

    // Kernels of one substep from state buffer c; ev (optional) receives
    // events after bin, p2g, grid (incl. an implicit phase-field solve), g2p.
    // Host bookkeeping is left alone.  host_checks: the implicit solve reads
    // its done flag every 4 iterations and stops launching (not when capturing).
    gmpm_status launch_one(cudaStream_t s, int c, cudaEvent_t* ev, bool host_checks = true,
                           int64_t* kernels = nullptr) {
        const LaunchCfg lc = cfg();
        const bool keys_ready = keys_fresh;
        keys_fresh = false;  // until this substep's G2P has keyed the new positions
        int64_t nk = (keys_ready ? kBinningKernelsKeysReady : kBinningKernels) + 4;
        GMPM_TRY(launch_binning<R>(d_sc, st[c], bin, scan, d_cnt, lc.num_sms, s, keys_ready));
        if (ev) GMPM_TRY(cudaEventRecord(ev[0], s));
        GMPM_TRY(launch_p2g<R>(d_sc, st[c], aux, bin, grid, d_cnt, lc, s));
        if (ev) GMPM_TRY(cudaEventRecord(ev[1], s));
        GMPM_TRY(launch_grid<R>(d_sc, bin, grid, d_cnt, lc, s));
        if (implicit_pf()) {
            GMPM_TRY(launch_pcg_init<R>(d_sc, bin, grid, d_cnt, lc, s));
            nk += kPcgInitKernels + kPcgFinishKernels;
            for (int it = 0; it < desc.pcg_max_iterations; ++it) {
                GMPM_TRY(launch_pcg_iteration<R>(d_sc, st[c], aux, bin, grid, d_cnt, lc, s));
                nk += kPcgIterationKernels;
                if (host_checks && (it & 3) == 3) {
                    GMPM_TRY(cudaMemcpyAsync(pcg_done_host, &grid.pcg.scal->done, sizeof(int),
                                             cudaMemcpyDeviceToHost, s));
                    GMPM_TRY(cudaStreamSynchronize(s));
                    if (*pcg_done_host) break;
                }
            }
            GMPM_TRY(launch_pcg_finish<R>(d_sc, bin, grid, d_cnt, lc, s));
        }
        if (kernels) *kernels = nk;
        if (ev) GMPM_TRY(cudaEventRecord(ev[2], s));
        GMPM_TRY(launch_g2p<R>(d_sc, d_sc64, desc.precision == GMPM_PRECISION_FP32_FP64SVD ? d_sc64 : nullptr,
                               st[c], st[1 - c], aux, bin, grid, d_cnt, lc, s));
        keys_fresh = true;
        if (ev) GMPM_TRY(cudaEventRecord(ev[3], s));
        return GMPM_OK;
    }

    gmpm_status one_substep(cudaStream_t s, cudaEvent_t* ev) {
        int64_t nk = 0;
        gmpm_status r = launch_one(s, cur, ev, true, &nk);
        if (r != GMPM_OK) return r;
        commit_substeps(1);
        launches += nk - kernels_per_substep();
        return GMPM_OK;
    }

    // batched stepping (SceneBase)
    uint64_t uid() const override { return uid_; }
    gmpm_context* context() const override { return ctx; }
    int64_t particles() const override { return n; }
    size_t device_bytes() const override { return dev_bytes_; }
    int parity() const override { return cur; }
    int kernels_per_substep() const override {
        return kBinningKernelsKeysReady + 4 +
               (implicit_pf() ? kPcgInitKernels + kPcgFinishKernels + desc.pcg_max_iterations * kPcgIterationKernels
                              : 0);
    }
    gmpm_status launch_substep(cudaStream_t s, int c) override {
        if (c != 0 && c != 1) return GMPM_INVALID_ARG;
        return launch_one(s, c, nullptr, false);
    }
    void commit_substeps(int nsub, bool own_launches = true) override {
        if (own_launches) launches += (int64_t)nsub * kernels_per_substep();  // as launched by a captured substep
        if (nsub & 1) cur = 1 - cur;
        binned = false;
    }
    void set_sm_share(int sms) override { share_ = sms > 0 ? sms : 0; }
    int sm_share() const override { return share_; }
    int batch_kind() const override {
        if (implicit_pf()) return -1;
        const LaunchCfg lc = cfg();
        return (sizeof(R) == 8 ? 8 : 0) | (desc.deterministic ? 4 : 0) | (lc.other_models ? 2 : 0) |
               (desc.precision == GMPM_PRECISION_FP32_FP64SVD ? 1 : 0);
    }
    void batch_args(int c, void* out) const override {
        SceneArgs<R>& a = *static_cast<SceneArgs<R>*>(out);
        a.sc = d_sc;
        a.sc64 = d_sc64;
        a.in = st[c];
        a.out = st[1 - c];
        a.aux = aux;
        a.bin = bin;
        a.grid = grid;
        a.cnt = d_cnt;
        a.scan = scan;
    }
    void batch_sizes(int64_t* n_out, uint32_t* key_space, int* nb_cap, int* ng_cap) const override {
        *n_out = n;
        *key_space = bin.key_space;
        *nb_cap = bin.nb_cap;
        *ng_cap = bin.ng_cap;
    }

    // ---- checkpoint ---------------------------------------------------------
    // Every particle plane of the current state, in the internal order, with
    // the clock; binning and grid are rebuilt by the next substep.
    template <typename F>
    void for_each_plane(int c, F&& f) {
        for (int a = 0; a < 3; ++a) f(st[c].x[a], sizeof(R));
        for (int k = 0; k < 3; ++k) f(st[c].fw[k], sizeof(Word4<R>));
        f(st[c].c, sizeof(R));
        f(st[c].m, sizeof(R));
        f(st[c].id, sizeof(uint32_t));
        for (int a = 0; a < 3; ++a) f(aux.v[a], sizeof(R));
        for (int q = 0; q < 9; ++q) f(aux.B[q], sizeof(R));
        for (int q = 0; q < 6; ++q) f(aux.sigma[q], sizeof(R));
        f(aux.vol, sizeof(R));
        f(aux.FP, sizeof(R));
        for (int a = 0; a < 3; ++a) f(aux.q[a], sizeof(R));
    }

    gmpm_status save(const char* path) override {
        GMPM_TRY(cudaSetDevice(ctx->device));
        GMPM_TRY(cudaDeviceSynchronize());
        SnapshotHeader h{};
        std::memcpy(h.magic, kSnapshotMagic, sizeof(h.magic));
        h.version = kSnapshotVersion;
        h.real_bytes = (uint32_t)sizeof(R);
        h.desc_bytes = (uint32_t)sizeof(gmpm_scene_desc);
        h.n = n;
        Counters c{};
        GMPM_TRY(cudaMemcpy(&c, d_cnt, sizeof(c), cudaMemcpyDeviceToHost));
        GMPM_TRY(cudaMemcpy(&h.dt, &d_sc64->dt, sizeof(double), cudaMemcpyDeviceToHost));
        h.time = c.time;
        h.substeps = c.substeps;
        FILE* f = std::fopen(path, "wb");
        if (!f) return GMPM_IO_ERROR;
        bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(&desc, sizeof(desc), 1, f) == 1;
        std::vector<unsigned char> buf((size_t)n * sizeof(Word4<double>));
        for_each_plane(cur, [&](const void* p, size_t esz) {
            if (!ok) return;
            ok = cudaMemcpy(buf.data(), p, (size_t)n * esz, cudaMemcpyDeviceToHost) == cudaSuccess &&
                 std::fwrite(buf.data(), esz, (size_t)n, f) == (size_t)n;
        });
        ok = (std::fclose(f) == 0) && ok;
        return ok ? GMPM_OK : GMPM_IO_ERROR;
    }

    // Overwrite the freshly created state with a snapshot's planes and clock.
    gmpm_status restore(FILE* f, const SnapshotHeader& h) {
        std::vector<unsigned char> buf((size_t)n * sizeof(Word4<double>));
        bool ok = true;
        for_each_plane(cur, [&](void* p, size_t esz) {
            if (!ok) return;
            ok = std::fread(buf.data(), esz, (size_t)n, f) == (size_t)n &&
                 cudaMemcpy(p, buf.data(), (size_t)n * esz, cudaMemcpyHostToDevice) == cudaSuccess;
        });
        if (!ok) return GMPM_IO_ERROR;
        Counters c{};
        GMPM_TRY(cudaMemcpy(&c, d_cnt, sizeof(c), cudaMemcpyDeviceToHost));
        c.time = h.time;
        c.substeps = h.substeps;
        GMPM_TRY(cudaMemcpy(d_cnt, &c, sizeof(c), cudaMemcpyHostToDevice));
        const R dtr = (R)h.dt;
        GMPM_TRY(cudaMemcpy(&d_sc->dt, &dtr, sizeof(R), cudaMemcpyHostToDevice));
        GMPM_TRY(cudaMemcpy(&d_sc64->dt, &h.dt, sizeof(double), cudaMemcpyHostToDevice));
        GMPM_TRY(refresh_keys(0));
        GMPM_TRY(cudaDeviceSynchronize());
        binned = false;
        return GMPM_OK;
    }

    gmpm_status substep(int nsteps, cudaStream_t s) override {
        if (nsteps < 0) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        for (int it = 0; it < nsteps; ++it) {
            gmpm_status r = one_substep(s, nullptr);
            if (r != GMPM_OK) return r;
        }
        return GMPM_OK;
    }

    gmpm_status substep_timed(int nsteps, cudaStream_t s, gmpm_stage_times* out) override {
        if (nsteps < 0 || !out) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        std::memset(out, 0, sizeof(*out));
        std::vector<cudaEvent_t> ev((size_t)nsteps * 5);
        for (auto& e : ev) GMPM_TRY(cudaEventCreate(&e));
        gmpm_status r = GMPM_OK;
        for (int it = 0; it < nsteps && r == GMPM_OK; ++it) {
            cudaEvent_t* e = &ev[(size_t)it * 5];
            cudaEventRecord(e[0], s);
            r = one_substep(s, e + 1);
        }
        cudaError_t ce = cudaEventSynchronize(ev.back());
        if (r == GMPM_OK && ce == cudaSuccess) {
            for (int it = 0; it < nsteps; ++it) {
                cudaEvent_t* e = &ev[(size_t)it * 5];
                float t[4];
                for (int q = 0; q < 4; ++q) cudaEventElapsedTime(&t[q], e[q], e[q + 1]);
                out->bin_ms += t[0];
                out->p2g_ms += t[1];
                out->grid_ms += t[2];
                out->g2p_ms += t[3];
                out->total_ms += t[0] + t[1] + t[2] + t[3];
            }
            out->substeps = nsteps;
        }
        for (auto& e : ev) cudaEventDestroy(e);
        if (r != GMPM_OK) return r;
        return cuda_status(ce);
    }

    gmpm_status rebin(cudaStream_t s) override {
        GMPM_TRY(cudaSetDevice(ctx->device));
        launches += kBinningKernels;
        return do_bin(s);
    }

    gmpm_status read_particles(int field, int dtype, int order, void* dst, size_t bytes, cudaStream_t s) override {
        const int nc = field_components(field);
        if (nc == 0 || !dst) return GMPM_INVALID_ARG;
        if (dtype < 0 || dtype > 2 || order < 0 || order > 1) return GMPM_INVALID_ARG;
        const size_t esz = dtype == GMPM_DTYPE_F64 ? 8 : 4;
        const size_t need = (size_t)n * nc * esz;
        if (bytes < need) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        cudaPointerAttributes attr{};
        bool on_device = false;
        if (cudaPointerGetAttributes(&attr, dst) == cudaSuccess)
            on_device = (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
        else
            cudaGetLastError();
        if (on_device) {
            GMPM_TRY(launch_pack_field<R>(st[cur], aux, field, dtype, order, n, dst, s));
            GMPM_TRY(cudaStreamSynchronize(s));
            return GMPM_OK;
        }
        if (staging_bytes < need) {
            if (staging) cudaFreeAsync(staging, s);
            staging = nullptr;
            staging_bytes = 0;
            GMPM_TRY(cudaMallocAsync(&staging, need, s));
            staging_bytes = need;
        }
        GMPM_TRY(launch_pack_field<R>(st[cur], aux, field, dtype, order, n, staging, s));
        GMPM_TRY(cudaMemcpyAsync(dst, staging, need, cudaMemcpyDefault, s));
        GMPM_TRY(cudaStreamSynchronize(s));
        return GMPM_OK;
    }

    // Ping-pong device staging for overlapped reads: a read packs on the
    // caller's stream into the buffer whose previous copy has finished, and
    // copies to the caller's memory on the copy stream.
    cudaStream_t copy_stream_ = nullptr;
    void* rstage_[2] = {nullptr, nullptr};
    size_t rstage_bytes_[2] = {0, 0};
    cudaEvent_t rstage_packed_[2] = {nullptr, nullptr}, rstage_free_[2] = {nullptr, nullptr};
    int rnext_ = 0;

    gmpm_status read_particles_async(int field, int dtype, int order, void* dst, size_t bytes,
                                     cudaStream_t s) override {
        const int nc = field_components(field);
        if (nc == 0 || !dst) return GMPM_INVALID_ARG;
        if (dtype < 0 || dtype > 2 || order < 0 || order > 1) return GMPM_INVALID_ARG;
        const size_t need = (size_t)n * nc * (dtype == GMPM_DTYPE_F64 ? 8 : 4);
        if (bytes < need) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        if (!copy_stream_) {
            GMPM_TRY(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
            for (int b = 0; b < 2; ++b) {
                GMPM_TRY(cudaEventCreateWithFlags(&rstage_packed_[b], cudaEventDisableTiming));
                GMPM_TRY(cudaEventCreateWithFlags(&rstage_free_[b], cudaEventDisableTiming));
                GMPM_TRY(cudaEventRecord(rstage_free_[b], copy_stream_));
            }
        }
        const int b = rnext_;
        rnext_ ^= 1;
        GMPM_TRY(cudaStreamWaitEvent(s, rstage_free_[b], 0));  // the buffer's previous copy has left
        if (rstage_bytes_[b] < need) {
            if (rstage_[b]) cudaFreeAsync(rstage_[b], s);
            rstage_[b] = nullptr;
            rstage_bytes_[b] = 0;
            GMPM_TRY(cudaMallocAsync(&rstage_[b], need, s));
            rstage_bytes_[b] = need;
        }
        GMPM_TRY(launch_pack_field<R>(st[cur], aux, field, dtype, order, n, rstage_[b], s));
        GMPM_TRY(cudaEventRecord(rstage_packed_[b], s));
        GMPM_TRY(cudaStreamWaitEvent(copy_stream_, rstage_packed_[b], 0));
        GMPM_TRY(cudaMemcpyAsync(dst, rstage_[b], need, cudaMemcpyDefault, copy_stream_));
        GMPM_TRY(cudaEventRecord(rstage_free_[b], copy_stream_));
        return GMPM_OK;
    }

    gmpm_status reads_wait() override {
        GMPM_TRY(cudaSetDevice(ctx->device));
        if (copy_stream_) GMPM_TRY(cudaStreamSynchronize(copy_stream_));
        return GMPM_OK;
    }

    gmpm_status read_binning(int array, void* dst, size_t bytes) override {
        if (!dst) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        GMPM_TRY(cudaDeviceSynchronize());
        Counters h{};
        GMPM_TRY(cudaMemcpy(&h, d_cnt, sizeof(h), cudaMemcpyDeviceToHost));
        const int64_t nb = std::min(h.n_blocks, bin.nb_cap), ng = std::min(h.n_grid_blocks, bin.ng_cap);
        auto copy = [&](const void* src, size_t sz) -> gmpm_status {
            if (bytes < sz) return GMPM_INVALID_ARG;
            GMPM_TRY(cudaMemcpy(dst, src, sz, cudaMemcpyDeviceToHost));
            return GMPM_OK;
        };
        switch (array) {
            case GMPM_BIN_COUNTS: {
                if (bytes < 4 * sizeof(int64_t)) return GMPM_INVALID_ARG;
                int64_t* o = reinterpret_cast<int64_t*>(dst);
                o[0] = n;
                o[1] = h.n_blocks;
                o[2] = h.n_grid_blocks;
                o[3] = bin.key_space;
                return GMPM_OK;
            }
            case GMPM_BIN_PERM: return copy(bin.perm, n * 4);
            case GMPM_BIN_KEYS: return copy(bin.keys_sorted, n * 4);
            case GMPM_BIN_BLOCK_KEYS: return copy(bin.block_keys, nb * 4);
            case GMPM_BIN_BLOCK_START: {
                if (bytes < (size_t)(nb + 1) * 4) return GMPM_INVALID_ARG;
                std::vector<int32_t> cs((size_t)nb * 64 + 1);
                GMPM_TRY(cudaMemcpy(cs.data(), bin.cell_start, cs.size() * 4, cudaMemcpyDeviceToHost));
                int32_t* o = reinterpret_cast<int32_t*>(dst);
                for (int64_t b = 0; b <= nb; ++b) o[b] = cs[b * 64];
                return GMPM_OK;
            }
            case GMPM_BIN_CELL_START: return copy(bin.cell_start, (nb * 64 + 1) * 4);
            case GMPM_BIN_GRID_KEYS: return copy(bin.grid_keys, ng * 4);
            case GMPM_BIN_ADJ: return copy(bin.adj, nb * 8 * 4);
            default: return GMPM_INVALID_ARG;
        }
    }

    gmpm_status diagnostics(gmpm_diag* out) override {
        if (!out) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        GMPM_TRY(launch_particle_diag<R>(st[cur], aux, n, d_pdiag, 0));
        GMPM_TRY(cudaDeviceSynchronize());
        double pd[8], gd[8];
        Counters h{};
        GMPM_TRY(cudaMemcpy(pd, d_pdiag, sizeof(pd), cudaMemcpyDeviceToHost));
        GMPM_TRY(cudaMemcpy(gd, grid.diag, sizeof(gd), cudaMemcpyDeviceToHost));
        GMPM_TRY(cudaMemcpy(&h, d_cnt, sizeof(h), cudaMemcpyDeviceToHost));
        std::memset(out, 0, sizeof(*out));
        out->particle_mass = pd[0];
        for (int a = 0; a < 3; ++a) {
            out->particle_momentum[a] = pd[1 + a];
            out->grid_momentum[a] = gd[1 + a];
        }
        out->grid_mass = gd[0];
        out->kinetic_energy = pd[4];
        out->max_speed = pd[5];
        out->min_damage = pd[6];
        out->time = h.time;
        out->substeps = h.substeps;
        out->n_particles = n;
        out->n_blocks = h.n_blocks;
        out->n_grid_blocks = h.n_grid_blocks;
        out->flags = h.flags;
        out->kernel_launches = launches;
        GMPM_TRY(cudaMemcpy(&out->dt, &d_sc64->dt, sizeof(double), cudaMemcpyDeviceToHost));
        out->pcg_iterations = h.pcg_iterations;
        return GMPM_OK;
    }

    gmpm_status set_dt(double dt, cudaStream_t s) override {
        if (!(dt > 0)) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        // dt is read by every kernel from the scene block; the 64-bit copy keeps
        // the FP64-fallback block consistent.  Host staging is pinned and
        // double-buffered with the velocity conditions' events.
        if (!dt_staging) GMPM_TRY(cudaMallocHost(reinterpret_cast<void**>(&dt_staging), 2 * sizeof(DtBlock)));
        if (!dt_done[0]) {
            GMPM_TRY(cudaEventCreateWithFlags(&dt_done[0], cudaEventDisableTiming));
            GMPM_TRY(cudaEventCreateWithFlags(&dt_done[1], cudaEventDisableTiming));
            GMPM_TRY(cudaEventRecord(dt_done[0], s));
            GMPM_TRY(cudaEventRecord(dt_done[1], s));
        }
        const int k = dt_next;
        dt_next ^= 1;
        GMPM_TRY(cudaEventSynchronize(dt_done[k]));
        dt_staging[k].r = (R)dt;
        dt_staging[k].d = dt;
        GMPM_TRY(cudaMemcpyAsync(&d_sc->dt, &dt_staging[k].r, sizeof(R), cudaMemcpyHostToDevice, s));
        GMPM_TRY(cudaMemcpyAsync(&d_sc64->dt, &dt_staging[k].d, sizeof(double), cudaMemcpyHostToDevice, s));
        // in adaptive mode dt is the upper bound of the CFL step
        GMPM_TRY(cudaMemcpyAsync(&d_sc->dt_max, &dt_staging[k].d, sizeof(double), cudaMemcpyHostToDevice, s));
        GMPM_TRY(cudaMemcpyAsync(&d_sc64->dt_max, &dt_staging[k].d, sizeof(double), cudaMemcpyHostToDevice, s));
        GMPM_TRY(cudaEventRecord(dt_done[k], s));
        desc.dt = dt;
        return GMPM_OK;
    }
    struct DtBlock {
        R r;
        double d;
    };
    DtBlock* dt_staging = nullptr;
    cudaEvent_t dt_done[2] = {nullptr, nullptr};
    int dt_next = 0;

    // Two pinned host staging blocks for velocity-condition updates, so an
    // update can be written while the previous copy is still in flight.
    VelocityConditions<R>* bc_staging = nullptr;  // [2]
    cudaEvent_t bc_done[2] = {nullptr, nullptr};
    int bc_next = 0;

    gmpm_status set_velocity_conditions(const gmpm_slab_bc* slabs, int ns, const gmpm_sphere_bc* spheres, int nsp,
                                        cudaStream_t s) override {
        if (ns < 0 || ns > GMPM_MAX_SLAB_BCS || nsp < 0 || nsp > GMPM_MAX_SPHERE_BCS) return GMPM_INVALID_ARG;
        if ((ns > 0 && !slabs) || (nsp > 0 && !spheres)) return GMPM_INVALID_ARG;
        for (int q = 0; q < ns; ++q)
            if (slabs[q].axis < 0 || slabs[q].axis > 2) return GMPM_INVALID_ARG;
        GMPM_TRY(cudaSetDevice(ctx->device));
        if (!bc_staging) {
            GMPM_TRY(cudaMallocHost(reinterpret_cast<void**>(&bc_staging), 2 * sizeof(*bc_staging)));
            GMPM_TRY(cudaEventCreateWithFlags(&bc_done[0], cudaEventDisableTiming));
            GMPM_TRY(cudaEventCreateWithFlags(&bc_done[1], cudaEventDisableTiming));
            GMPM_TRY(cudaEventRecord(bc_done[0], s));
            GMPM_TRY(cudaEventRecord(bc_done[1], s));
        }
        const int k = bc_next;
        bc_next ^= 1;
        GMPM_TRY(cudaEventSynchronize(bc_done[k]));  // the copy that last read block k has left
        fill_velocity_conditions<R>(slabs, ns, spheres, nsp, bc_staging[k]);
        GMPM_TRY(cudaMemcpyAsync(&d_sc->bc, &bc_staging[k], sizeof(VelocityConditions<R>), cudaMemcpyHostToDevice, s));
        GMPM_TRY(cudaEventRecord(bc_done[k], s));
        desc.n_slab_bcs = ns;
        desc.n_sphere_bcs = nsp;
        for (int q = 0; q < ns; ++q) desc.slabs[q] = slabs[q];
        for (int q = 0; q < nsp; ++q) desc.spheres[q] = spheres[q];
        return GMPM_OK;
    }

    gmpm_status status_on_stream(cudaStream_t s) override {
        GMPM_TRY(cudaSetDevice(ctx->device));
        Counters h{};
        GMPM_TRY(cudaMemcpyAsync(&h, d_cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
        GMPM_TRY(cudaStreamSynchronize(s));
        return flags_status(h.flags);
    }
    gmpm_status enqueue_flags(unsigned int* dst, cudaStream_t s) override {
        GMPM_TRY(cudaMemcpyAsync(dst, &d_cnt->flags, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
        return GMPM_OK;
    }
    gmpm_status enqueue_read(int field, int dtype, int order, void* dst, cudaStream_t s) override {
        const int nc = field_components(field);
        if (nc == 0 || !dst || dtype < 0 || dtype > 2 || order < 0 || order > 1) return GMPM_INVALID_ARG;
        const size_t need = (size_t)n * nc * (dtype == GMPM_DTYPE_F64 ? 8 : 4);
        if (staging_bytes < need) {
            if (staging) cudaFreeAsync(staging, s);
            staging = nullptr;
            staging_bytes = 0;
            GMPM_TRY(cudaMallocAsync(&staging, need, s));
            staging_bytes = need;
        }
        GMPM_TRY(launch_pack_field<R>(st[cur], aux, field, dtype, order, n, staging, s));
        GMPM_TRY(cudaMemcpyAsync(dst, staging, need, cudaMemcpyDefault, s));
        return GMPM_OK;
    }

    gmpm_status sync() override {
        GMPM_TRY(cudaSetDevice(ctx->device));
        GMPM_TRY(cudaDeviceSynchronize());
        Counters h{};
        GMPM_TRY(cudaMemcpy(&h, d_cnt, sizeof(h), cudaMemcpyDeviceToHost));
        if (h.flags & GMPM_FLAG_COPY_TIMEOUT) return GMPM_CUDA_ERROR;
        if (h.flags & GMPM_FLAG_TABLE_OVERFLOW) return GMPM_TABLE_OVERFLOW;
        if (h.flags & GMPM_FLAG_OUT_OF_DOMAIN) return GMPM_OUT_OF_DOMAIN;
        if (h.flags & GMPM_FLAG_NONFINITE) return GMPM_NONFINITE;
        return GMPM_OK;
    }
};

}  // namespace gmpm

// ---- key-only helpers used at creation (declared in Scene) ----------------
namespace gmpm {
template <typename R>
void Scene<R>::launch_keys_only(cudaStream_t s) {
    launch_keys<R>(d_sc, st[cur], bin, d_cnt, s);
}
template <typename R>
void Scene<R>::mark_grid(cudaStream_t s) {
    launch_mark_grid(bin, s);
}
}  // namespace gmpm

extern "C" {

const char* gmpm_status_string(gmpm_status s) {
    switch (s) {
        case GMPM_OK: return "ok";
        case GMPM_INVALID_ARG: return "invalid argument";
        case GMPM_OOM: return "out of device memory";
        case GMPM_TABLE_OVERFLOW: return "page table capacity exceeded";
        case GMPM_NONFINITE: return "non-finite particle state";
        case GMPM_OUT_OF_DOMAIN: return "particle stencil outside the grid";
        case GMPM_CUDA_ERROR: return "CUDA error";
        case GMPM_NOT_SUPPORTED: return "not supported";
        case GMPM_NO_DEVICE: return "no CUDA device";
        case GMPM_IO_ERROR: return "checkpoint file error";
        default: return "unknown status";
    }
}

gmpm_status gmpm_context_create(int device, gmpm_context** out) {
    if (!out) return GMPM_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        return GMPM_NO_DEVICE;
    }
    if (device < 0 || device >= count) return GMPM_INVALID_ARG;
    gmpm_context* c = new (std::nothrow) gmpm_context();
    if (!c) return GMPM_OOM;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&c->prop, device) != cudaSuccess) {
        delete c;
        return GMPM_CUDA_ERROR;
    }
    c->num_sms = c->prop.multiProcessorCount;
    // Scenes allocate from the device's stream-ordered pool; keep freed memory
    // cached in the pool (this process only) so scenes created after others
    // were released reuse it without returning to the driver.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    *out = c;
    return GMPM_OK;
}

gmpm_status gmpm_context_destroy(gmpm_context* ctx) {
    if (!ctx) return GMPM_INVALID_ARG;
    delete ctx;
    return GMPM_OK;
}

gmpm_status gmpm_scene_desc_reference_defaults(gmpm_scene_desc* d, double dx, int rx, int ry, int rz) {
    if (!d || !(dx > 0)) return GMPM_INVALID_ARG;
    std::memset(d, 0, sizeof(*d));
    d->dx = dx;
    d->grid_res[0] = rx;
    d->grid_res[1] = ry;
    d->grid_res[2] = rz;
    d->dt = 1e-4;                                  // Simulator.cpp:172
    d->gravity[1] = -10.0;                         // TimeIntegrator.cu:100
    d->particle_volume = dx * dx * dx / 8.0;
    d->n_materials = 1;
    gmpm_material& m = d->materials[0];
    m.youngs_modulus = 2e2;                        // Simulator.cpp:114-116 (scene 1)
    m.poisson_ratio = 0.4;
    m.density = 3.0;
    m.yield_stress = 800.0;                        // ExplicitTimeIntegrator.cu:188
    m.hardening_law = GMPM_HARDENING_EXPONENTIAL;
    m.hardening = 3.0;                             // :189
    m.alpha_cap = 1.0;                             // :194
    m.dlambda_cap = 100.0;                         // :217-220
    m.strain_cap = 3.0;                            // :267-271
    m.psi_cap = 1e6;                               // :313
    m.fracture_energy = 3.0;                       // :317
    m.softening_onset = 0.01;                      // :320
    m.residual_fracture = 0.1;                     // :327
    m.theta = (double)0.0001f;                     // :334 (float)
    m.length_scale = 0.5 * dx;                     // :335
    m.mobility = 50.0;                             // Materials.cpp:13
    d->wall_bc = 1;
    d->wall_layers = 4;
    d->precision = GMPM_PRECISION_FP32;
    d->phase_field = GMPM_PHASE_FIELD_EXPLICIT;
    d->deterministic = 1;
    d->svd_fallback_ratio = 1e-3;
    d->adaptive_dt = 0;
    d->cfl_number = (double)0.3f;                  // Simulator.cpp:211
    d->pcg_max_iterations = 100;                   // ExplicitTimeIntegrator.cu:925
    d->pcg_max_combine = 0;
    d->pcg_tolerance = (double)1e-6f;              // :926 (float literal)
    return GMPM_OK;
}

gmpm_status gmpm_scene_create(gmpm_context* ctx, const gmpm_scene_desc* desc, const gmpm_particle_init* init,
                              gmpm_scene** out) {
    if (!ctx || !out) return GMPM_INVALID_ARG;
    *out = nullptr;
    gmpm_status v = gmpm::validate(desc, init);
    if (v != GMPM_OK) return v;
    gmpm_scene* s = new (std::nothrow) gmpm_scene();
    if (!s) return GMPM_OOM;
    gmpm_status r;
    if (desc->precision == GMPM_PRECISION_FP64) {
        auto* impl = new (std::nothrow) gmpm::Scene<double>();
        s->impl = impl;
        r = impl ? impl->create(ctx, desc, init) : GMPM_OOM;
    } else {
        auto* impl = new (std::nothrow) gmpm::Scene<float>();
        s->impl = impl;
        r = impl ? impl->create(ctx, desc, init) : GMPM_OOM;
    }
    if (r != GMPM_OK) {
        delete s->impl;
        delete s;
        cudaGetLastError();
        return r;
    }
    *out = s;
    return GMPM_OK;
}

gmpm_status gmpm_scene_save(gmpm_scene* s, const char* path) {
    if (!s || !path) return GMPM_INVALID_ARG;
    return s->impl->save(path);
}

gmpm_status gmpm_scene_load(gmpm_context* ctx, const char* path, gmpm_scene** out) {
    using namespace gmpm;
    if (!ctx || !path || !out) return GMPM_INVALID_ARG;
    *out = nullptr;
    FILE* f = std::fopen(path, "rb");
    if (!f) return GMPM_IO_ERROR;
    struct Closer {
        FILE* f;
        ~Closer() { std::fclose(f); }
    } closer{f};
    SnapshotHeader h{};
    gmpm_scene_desc desc{};
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kSnapshotMagic, 8) != 0 ||
        h.version != kSnapshotVersion || h.desc_bytes != sizeof(gmpm_scene_desc) || h.n <= 0 ||
        std::fread(&desc, sizeof(desc), 1, f) != 1)
        return GMPM_IO_ERROR;
    const size_t rb = desc.precision == GMPM_PRECISION_FP64 ? 8 : 4;
    if (h.real_bytes != rb) return GMPM_IO_ERROR;
    const long base = std::ftell(f);
    const int64_t n = h.n;
    // positions (planes 0-2), mass (plane 16) and ids (plane 17, counted in
    // real-sized planes: x 3, the three words 12, c 1, m 1) build the scene;
    // then every plane is restored over it
    std::vector<double> pos((size_t)n * 3), mass((size_t)n);
    std::vector<int32_t> mat((size_t)n);
    {
        std::vector<unsigned char> buf((size_t)n * rb);
        auto read_plane = [&](int64_t plane_index, std::vector<double>& dst, int stride, int comp) -> bool {
            if (std::fseek(f, base + (long)(plane_index * n * (int64_t)rb), SEEK_SET) != 0) return false;
            if (std::fread(buf.data(), rb, (size_t)n, f) != (size_t)n) return false;
            for (int64_t p = 0; p < n; ++p)
                dst[(size_t)(p * stride + comp)] =
                    rb == 8 ? reinterpret_cast<const double*>(buf.data())[p] : reinterpret_cast<const float*>(buf.data())[p];
            return true;
        };
        for (int a = 0; a < 3; ++a)
            if (!read_plane(a, pos, 3, a)) return GMPM_IO_ERROR;
        if (!read_plane(16, mass, 1, 0)) return GMPM_IO_ERROR;
        std::vector<uint32_t> ids((size_t)n);
        if (std::fseek(f, base + (long)(17 * n * (int64_t)rb), SEEK_SET) != 0 ||
            std::fread(ids.data(), 4, (size_t)n, f) != (size_t)n)
            return GMPM_IO_ERROR;
        for (int64_t p = 0; p < n; ++p) mat[(size_t)p] = (int32_t)(ids[(size_t)p] >> 28);
    }
    gmpm_particle_init init{n, pos.data(), nullptr, mass.data(), mat.data()};
    gmpm_scene* sc = nullptr;
    gmpm_status r = gmpm_scene_create(ctx, &desc, &init, &sc);
    if (r != GMPM_OK) return r;
    std::fseek(f, base, SEEK_SET);
    if (desc.precision == GMPM_PRECISION_FP64)
        r = static_cast<Scene<double>*>(sc->impl)->restore(f, h);
    else
        r = static_cast<Scene<float>*>(sc->impl)->restore(f, h);
    if (r != GMPM_OK) {
        gmpm_scene_destroy(sc);
        return r;
    }
    *out = sc;
    return GMPM_OK;
}

gmpm_status gmpm_scene_destroy(gmpm_scene* s) {
    if (!s) return GMPM_INVALID_ARG;
    delete s->impl;
    delete s;
    return GMPM_OK;
}

gmpm_status gmpm_substep(gmpm_scene* s, int n, void* stream) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->substep(n, reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_substep_timed(gmpm_scene* s, int n, void* stream, gmpm_stage_times* out) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->substep_timed(n, reinterpret_cast<cudaStream_t>(stream), out);
}

gmpm_status gmpm_rebin(gmpm_scene* s, void* stream) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->rebin(reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_scene_sync(gmpm_scene* s) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->sync();
}

gmpm_status gmpm_read_particles(gmpm_scene* s, int field, int dtype, int order, void* dst, size_t bytes,
                                void* stream) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->read_particles(field, dtype, order, dst, bytes, reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_read_particles_async(gmpm_scene* s, int field, int dtype, int order, void* dst, size_t bytes,
                                      void* stream) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->read_particles_async(field, dtype, order, dst, bytes, reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_read_wait(gmpm_scene* s) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->reads_wait();
}

gmpm_status gmpm_set_dt(gmpm_scene* s, double dt, void* stream) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->set_dt(dt, reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_set_velocity_conditions(gmpm_scene* s, const gmpm_slab_bc* slabs, int n_slabs,
                                         const gmpm_sphere_bc* spheres, int n_spheres, void* stream) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->set_velocity_conditions(slabs, n_slabs, spheres, n_spheres, reinterpret_cast<cudaStream_t>(stream));
}

gmpm_status gmpm_read_binning(gmpm_scene* s, int array, void* dst, size_t bytes) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->read_binning(array, dst, bytes);
}

gmpm_status gmpm_diagnostics(gmpm_scene* s, gmpm_diag* out) {
    if (!s) return GMPM_INVALID_ARG;
    return s->impl->diagnostics(out);
}

}  // extern "C"
