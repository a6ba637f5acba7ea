// C++ host side over the gmpm C-ABI, with the class and method names of the
// reference's host interface: MPMSimulator (GPU_MPM/Simulator.h:12-69),
// MPMTimeIntegrator / ExplicitTimeIntegrator (GPU_MPM/TimeIntegrator.cuh:11-62),
// Particles (GPU_MPM/Particles.cuh:7-75), SPGrid (GPU_MPM/SPGrid.h:3-36),
// DomainTransformer (GPU_MPM/Transformer.cuh:9-51) and Model
// (GPU_MPM/Models.h:9-30).  Header-only; link against libgmpm.so.
//
// Error behaviour: where the reference prints and calls exit(0) on a CUDA
// error (GPU_MPM/cuda_tools.h:25-36), these classes throw GmpmError carrying
// the gmpm_status; build() returns false instead of throwing.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gmpm.h"

// Setting.h:40-44
struct vector3T {
    double x;
    double y;
    double z;
};

class GmpmError : public std::runtime_error {
  public:
    GmpmError(gmpm_status s, const std::string& what)
        : std::runtime_error(what + ": " + gmpm_status_string(s)), status(s) {}
    gmpm_status status;
};

inline void gmpm_check(gmpm_status s, const char* what) {
    if (s != GMPM_OK) throw GmpmError(s, what);
}

// Scene sampling (GPU_MPM/LoadSample.h:10-24) over gmpm_sample_*: the same
// particles as the reference's Sample, bit for bit.  The reference's grid
// resolution N comes from Setting.h (256); here it is the constructor's.
class Sample {
  public:
    explicit Sample(unsigned n_grid = 256) : N(n_grid) {}
    std::vector<vector3T> readObj(std::string fileName) const {
        return take([&](int64_t* n, double* p, int64_t cap) { return gmpm_sample_obj(fileName.c_str(), n, p, cap); },
                    "gmpm_sample_obj");
    }
    std::vector<vector3T> Initialize_Data_cube() const {
        return take([&](int64_t* n, double* p, int64_t cap) { return gmpm_sample_cube((int32_t)N, n, p, cap); },
                    "gmpm_sample_cube");
    }
    // Draws from the C library's rand() after srand(seed) (seed 1: the reference's run).
    std::vector<vector3T> Initial_data(unsigned int* center, unsigned int* res, std::string fileName,
                                       unsigned seed = 1) const {
        const uint32_t c[3] = {center[0], center[1], center[2]}, r[3] = {res[0], res[1], res[2]};
        return take(
            [&](int64_t* n, double* p, int64_t cap) {
                return gmpm_sample_sdf(fileName.c_str(), c, r, 1.0 / N, seed, n, p, cap);
            },
            "gmpm_sample_sdf");
    }
    unsigned N;

  private:
    template <class F>
    static std::vector<vector3T> take(F call, const char* what) {
        int64_t n = 0;
        gmpm_check(call(&n, nullptr, 0), what);
        std::vector<vector3T> out((size_t)n);
        static_assert(sizeof(vector3T) == 3 * sizeof(double), "vector3T is three doubles");
        gmpm_check(call(&n, reinterpret_cast<double*>(out.data()), n), what);
        return out;
    }
};

// Material (GPU_MPM/Materials.h:15-23): constants live in the scene.
class ElasticMaterial {
  public:
    explicit ElasticMaterial(const gmpm_material& m) : mat(m) {
        const double E = m.youngs_modulus, nu = m.poisson_ratio;
        _youngsModulus = E;
        _poissonRatio = nu;
        _density = m.density;
        _lambda = E * nu / ((1 + nu) * (1 - 2 * nu));
        _mu = E / (2 * (1 + nu));
        _kappa = E / (3 * (1 - 2 * nu));
        parabolic_M = m.mobility;
    }
    gmpm_material mat;
    double _youngsModulus, _poissonRatio, _density, _lambda, _mu, _kappa, parabolic_M;
};

// Particles (GPU_MPM/Particles.cuh:7-75): a view of the scene's particles.
class Particles {
  public:
    Particles(gmpm_scene* s, unsigned int n) : scene_(s), _numParticle(n) {}
    // Positions, velocities and original indices in the current sorted order
    // (Particles.cpp:33-52 copies d_pos in sorted order).
    void Attribs_Back_Host(std::vector<vector3T>& h_pos, std::vector<vector3T>& h_vel,
                           std::vector<unsigned int>& h_indices) {
        h_pos.resize(_numParticle);
        h_vel.resize(_numParticle);
        h_indices.resize(_numParticle);
        gmpm_check(gmpm_read_particles(scene_, GMPM_FIELD_POSITION, GMPM_DTYPE_F64, GMPM_ORDER_INTERNAL,
                                       h_pos.data(), h_pos.size() * sizeof(vector3T), nullptr),
                   "Attribs_Back_Host(position)");
        gmpm_check(gmpm_read_particles(scene_, GMPM_FIELD_VELOCITY, GMPM_DTYPE_F64, GMPM_ORDER_INTERNAL,
                                       h_vel.data(), h_vel.size() * sizeof(vector3T), nullptr),
                   "Attribs_Back_Host(velocity)");
        std::vector<int32_t> ids(_numParticle);
        gmpm_check(gmpm_read_particles(scene_, GMPM_FIELD_ID, GMPM_DTYPE_I32, GMPM_ORDER_INTERNAL, ids.data(),
                                       ids.size() * sizeof(int32_t), nullptr),
                   "Attribs_Back_Host(id)");
        for (unsigned int p = 0; p < _numParticle; ++p) h_indices[p] = (unsigned int)ids[p];
    }
    // Damage (the reference copies d_phase_C next to the positions).
    void Phase_Back_Host(std::vector<double>& h_phase) {
        h_phase.resize(_numParticle);
        gmpm_check(gmpm_read_particles(scene_, GMPM_FIELD_DAMAGE, GMPM_DTYPE_F64, GMPM_ORDER_INTERNAL,
                                       h_phase.data(), h_phase.size() * sizeof(double), nullptr),
                   "Phase_Back_Host");
    }
    // Particle_kernal.cu:421-440: squared maximum particle speed.
    void getMaxParticleVel_c(double* maxVelSquared) {
        gmpm_diag d;
        gmpm_check(gmpm_diagnostics(scene_, &d), "getMaxParticleVel_c");
        *maxVelSquared = d.max_speed * d.max_speed;
    }
    // Particle_kernal.cu:484-542 (sort) + Transformer.cpp:71-82 (rebuild).
    void sort_by_offsets() { gmpm_check(gmpm_rebin(scene_, nullptr), "sort_by_offsets"); }
    // Particle_kernal.cu:544-573: here G2P writes the new order while it reads
    // the old one, so there is nothing left to do.
    void reorder() {}

  private:
    gmpm_scene* scene_;

  public:
    unsigned int _numParticle;
};

// SPGrid (GPU_MPM/SPGrid.h:3-36): pages are rebuilt every substep from the
// particles; the grid result is transient and needs no clearing.
class SPGrid {
  public:
    SPGrid(double dc, const int res[3]) : _dc(dc), _width(res[0]), _height(res[1]), _depth(res[2]) {}
    void clear() {}
    double _dc;
    int _width, _height, _depth;
};

// DomainTransformer (GPU_MPM/Transformer.cuh:9-51).
class DomainTransformer {
  public:
    explicit DomainTransformer(gmpm_scene* s) : scene_(s) {}
    void rebuild() { gmpm_check(gmpm_rebin(scene_, nullptr), "rebuild"); }
    // Counts after the last binning: _numPage (active pages), _numTotalPage
    // (with the + neighbour pages).
    void counts(int* numPage, int* numTotalPage) {
        int64_t c[4];
        gmpm_check(gmpm_read_binning(scene_, GMPM_BIN_COUNTS, c, sizeof(c)), "counts");
        *numPage = (int)c[1];
        *numTotalPage = (int)c[2];
    }

  private:
    gmpm_scene* scene_;
};

// Model (GPU_MPM/Models.h:9-30).
class Model {
  public:
    Model(std::unique_ptr<Particles> p, std::unique_ptr<ElasticMaterial> m)
        : _particle(std::move(p)), _material(std::move(m)) {}
    std::unique_ptr<Particles>& getParticlesPtr() { return _particle; }
    std::unique_ptr<ElasticMaterial>& getMaterialPtr() { return _material; }

  private:
    std::unique_ptr<Particles> _particle;
    std::unique_ptr<ElasticMaterial> _material;
};

// MPMTimeIntegrator (GPU_MPM/TimeIntegrator.cuh:11-44).
class MPMTimeIntegrator {
  public:
    virtual ~MPMTimeIntegrator() {}
    virtual void integrate(int type, float* simulationTime, float* preprocessTime, const double dt, Model& model,
                           std::unique_ptr<SPGrid>& grid, std::unique_ptr<DomainTransformer>& trans) = 0;
};

// ExplicitTimeIntegrator (GPU_MPM/TimeIntegrator.cuh:47-61,
// ExplicitTimeIntegrator.cu:881-994).  simulationTime receives the device
// time of P2G + grid + G2P, preprocessTime the binning, as the reference's
// events split them.
class ExplicitTimeIntegrator : public MPMTimeIntegrator {
  public:
    explicit ExplicitTimeIntegrator(gmpm_scene* s, double dt) : scene_(s), dt_(dt) {}
    void integrate(int, float* simulationTime, float* preprocessTime, const double dt, Model&,
                   std::unique_ptr<SPGrid>&, std::unique_ptr<DomainTransformer>&) override {
        if (dt != dt_) {
            gmpm_check(gmpm_set_dt(scene_, dt, nullptr), "integrate(set_dt)");
            dt_ = dt;
        }
        gmpm_stage_times t;
        gmpm_check(gmpm_substep_timed(scene_, 1, nullptr, &t), "integrate");
        if (simulationTime) *simulationTime = (float)(t.p2g_ms + t.grid_ms + t.g2p_ms);
        if (preprocessTime) *preprocessTime = (float)t.bin_ms;
    }

  private:
    gmpm_scene* scene_;
    double dt_;
};

// MPMSimulator (GPU_MPM/Simulator.h:12-69, Simulator.cpp).
class MPMSimulator {
  public:
    MPMSimulator() : _currentFrame(0), _currentTime(0.0), _frameRate(48.0) {}
    ~MPMSimulator() { release(); }
    MPMSimulator(const MPMSimulator&) = delete;
    MPMSimulator& operator=(const MPMSimulator&) = delete;

    // Simulator.cpp:76-198.  The reference's scenes sample assets that are not
    // shipped; buildtype selects the synthetic benchmark scenes instead:
    //   0 = notched bar (16x16x64 cells, dx = 1/128, 8 ppc, pulled at +/-0.5 m/s)
    //   1 = four stacked plates (256x256x16 cells each, dx = 1/256, 8 ppc,
    //       sphere impactor at 5 m/s, gravity -9.8)
    //   2 = the plate scene at 8,388,608 particles (128x128x16 cells, dx = 1/128)
    bool build(unsigned int buildtype, int device = 0) {
        try {
            release();
            gmpm_check(gmpm_context_create(device, &ctx_), "context_create");
            gmpm_scene_desc d;
            std::vector<double> pos, mass, vel;
            std::vector<int32_t> mat;
            if (buildtype == 0)
                notched_bar(d, pos, mat);
            else if (buildtype == 1 || buildtype == 2)
                plates(d, pos, mat, buildtype == 1 ? 256 : 128, buildtype == 1 ? 1.0 / 256 : 1.0 / 128,
                       buildtype == 1 ? 8 : 4, buildtype == 1 ? 160 : 96);
            else
                return false;
            return build(d, pos, mat);
        } catch (const GmpmError&) {
            release();
            return false;
        }
    }

    // Generic form: any scene description and particle set.
    bool build(const gmpm_scene_desc& d, const std::vector<double>& positions, const std::vector<int32_t>& mat_ids,
               const std::vector<double>* velocities = nullptr) {
        try {
            if (!ctx_) gmpm_check(gmpm_context_create(0, &ctx_), "context_create");
            numParticle = (unsigned int)(positions.size() / 3);
            std::vector<double> mass(numParticle, d.materials[0].density * d.particle_volume);
            gmpm_particle_init init;
            init.count = numParticle;
            init.positions = positions.data();
            init.velocities = velocities ? velocities->data() : nullptr;
            init.masses = mass.data();
            init.material_ids = mat_ids.empty() ? nullptr : mat_ids.data();
            gmpm_check(gmpm_scene_create(ctx_, &d, &init, &scene_), "scene_create");
            desc_ = d;
            _dtDefault = d.dt;
            h_pGrid = std::make_unique<SPGrid>(d.dx, d.grid_res);
            h_pTrans = std::make_unique<DomainTransformer>(scene_);
            h_pTimeIntegrator = std::make_unique<ExplicitTimeIntegrator>(scene_, d.dt);
            h_models.clear();
            h_models.emplace_back(std::make_unique<Particles>(scene_, numParticle),
                                  std::make_unique<ElasticMaterial>(d.materials[0]));
            h_pos.assign(positions.size() / 3, vector3T{0, 0, 0});
            for (unsigned int p = 0; p < numParticle; ++p)
                h_pos[p] = vector3T{positions[3 * p], positions[3 * p + 1], positions[3 * p + 2]};
            return true;
        } catch (const GmpmError&) {
            release();
            return false;
        }
    }

    // Simulator.cpp:200-225: dt = min(dt_default, 0.3 dx / v_max).
    double computeDt(const double /*cur*/, const double /*next*/) {
        double dt = _dtDefault, maxVel = 0;
        getModelParticlePtr()->getMaxParticleVel_c(&maxVel);
        maxVel = std::sqrt(maxVel);
        if (maxVel > 0 && (maxVel = desc_.dx * 0.3 / maxVel) < _dtDefault) dt = maxVel;
        return dt;
    }

    // Simulator.cpp:227-259: one substep per frame, then positions back to the host.
    void simulateStick(float* cflTime, float* preTime, float* simuTime, int type) {
        const double dt = computeDt(_currentTime, _currentFrame / _frameRate);
        if (cflTime) *cflTime = 0.f;
        if (dt > 0.0) getTimeIntegratorPtr()->integrate(type, simuTime, preTime, dt, getModel(0), h_pGrid, h_pTrans);
        _currentTime += dt;
        _currentFrame++;
        getModelParticlePtr()->Attribs_Back_Host(h_pos, h_vel, h_indices);
    }

    // Simulator.h:35 declares writePartio without a definition; here it writes
    // a restartable checkpoint of the scene (gmpm_scene_save; gmpm_scene_load
    // resumes it bitwise).
    void writePartio(const std::string& filename) {
        gmpm_check(gmpm_scene_save(scene_, filename.c_str()), "writePartio");
    }

    std::unique_ptr<MPMTimeIntegrator>& getTimeIntegratorPtr() { return h_pTimeIntegrator; }
    std::unique_ptr<SPGrid>& getGridPtr() { return h_pGrid; }
    std::unique_ptr<DomainTransformer>& getTransformerPtr() { return h_pTrans; }
    Model& getModel(const unsigned int modelId = 0) { return h_models[modelId]; }
    std::unique_ptr<Particles>& getModelParticlePtr(const unsigned int modelId = 0) {
        return getModel(modelId).getParticlesPtr();
    }
    std::unique_ptr<ElasticMaterial>& getModelMaterialPtr(const unsigned int modelId = 0) {
        return getModel(modelId).getMaterialPtr();
    }
    gmpm_scene* scene() { return scene_; }

    std::vector<vector3T> h_pos;
    unsigned int numParticle = 0;

  private:
    void release() {
        h_models.clear();
        h_pTimeIntegrator.reset();
        h_pTrans.reset();
        h_pGrid.reset();
        if (scene_) gmpm_scene_destroy(scene_);
        scene_ = nullptr;
        if (ctx_) gmpm_context_destroy(ctx_);
        ctx_ = nullptr;
    }

    static void config_material(gmpm_material& m, double dx, double E) {
        m.youngs_modulus = E;
        m.poisson_ratio = 0.3;
        m.density = 1000.0;
        m.yield_stress = 200.0;
        m.hardening_law = GMPM_HARDENING_LINEAR;
        m.hardening = 0.1 * E;
        m.length_scale = 2.0 * dx;
        m.softening_onset = 0.05 / 2.0;
    }

    static void generate(const gmpm_scene_geometry& g, std::vector<double>& pos, std::vector<int32_t>& mat) {
        int64_t n = 0;
        gmpm_check(gmpm_generate_particles(&g, &n, nullptr, nullptr, 0), "generate_particles");
        pos.resize(3 * n);
        mat.resize(n);
        gmpm_check(gmpm_generate_particles(&g, &n, pos.data(), mat.data(), n), "generate_particles");
    }

    static void notched_bar(gmpm_scene_desc& d, std::vector<double>& pos, std::vector<int32_t>& mat) {
        const double dx = 1.0 / 128;
        const int res = 128, nx = 16, ny = 16, nz = 64;
        gmpm_scene_geometry g{};
        g.kind = 0;
        g.cells[0] = nx;
        g.cells[1] = ny;
        g.cells[2] = nz;
        g.ppc = 8;
        g.n_plates = 1;
        g.notch_width = 1;
        g.notch_depth = 4;
        g.dx = dx;
        g.origin[0] = (res - nx) / 2 * dx;
        g.origin[1] = (res - ny) / 2 * dx;
        g.origin[2] = (res - nz) / 2 * dx;
        g.seed = 0;
        generate(g, pos, mat);
        gmpm_check(gmpm_scene_desc_reference_defaults(&d, dx, res, res, res), "reference_defaults");
        d.dt = 1e-4;
        d.gravity[0] = d.gravity[1] = d.gravity[2] = 0.0;
        d.particle_volume = dx * dx * dx / 8;
        config_material(d.materials[0], dx, 1e5);
        const double z0 = g.origin[2], z1 = g.origin[2] + nz * dx;
        d.n_slab_bcs = 2;
        d.slabs[0].axis = 2;
        d.slabs[0].lo = 0.0;
        d.slabs[0].hi = z0 + 2 * dx;
        d.slabs[0].velocity[2] = -0.5;
        d.slabs[1].axis = 2;
        d.slabs[1].lo = z1 - 2 * dx;
        d.slabs[1].hi = res * dx;
        d.slabs[1].velocity[2] = 0.5;
    }

    static void plates(gmpm_scene_desc& d, std::vector<double>& pos, std::vector<int32_t>& mat, int cells, double dx,
                       int gap, int res_y) {
        const int margin = 8, thick = 16, n_plates = 4;
        const int res_xz = cells + 2 * margin;
        gmpm_scene_geometry g{};
        g.kind = 1;
        g.cells[0] = cells;
        g.cells[1] = thick;
        g.cells[2] = cells;
        g.ppc = 8;
        g.n_plates = n_plates;
        g.gap_cells = gap;
        g.dx = dx;
        g.origin[0] = g.origin[1] = g.origin[2] = margin * dx;
        g.seed = 0;
        generate(g, pos, mat);
        gmpm_check(gmpm_scene_desc_reference_defaults(&d, dx, res_xz, res_y, res_xz), "reference_defaults");
        d.dt = 5e-5;
        d.gravity[0] = 0.0;
        d.gravity[1] = -9.8;
        d.gravity[2] = 0.0;
        d.particle_volume = dx * dx * dx / 8;
        d.n_materials = n_plates;
        // E log-uniform in [5e4, 5e5] per plate (fixed draws of the benchmark scene)
        const double E[4] = {216736.318261958, 93058.64360568293, 54946.942117665036, 51939.48508933595};
        for (int k = 1; k < n_plates; ++k) d.materials[k] = d.materials[0];
        for (int k = 0; k < n_plates; ++k) config_material(d.materials[k], dx, E[k]);
        const double top = margin * dx + (n_plates * thick + (n_plates - 1) * gap) * dx;
        d.n_sphere_bcs = 1;
        d.spheres[0].center[0] = d.spheres[0].center[2] = res_xz * dx / 2;
        d.spheres[0].center[1] = top + 0.1 + 2 * dx;
        d.spheres[0].radius = 0.1;
        d.spheres[0].velocity[1] = -5.0;
    }

    gmpm_context* ctx_ = nullptr;
    gmpm_scene* scene_ = nullptr;
    gmpm_scene_desc desc_{};
    unsigned int _currentFrame;
    double _currentTime;
    double _frameRate;
    double _dtDefault = 1e-4;
    std::unique_ptr<SPGrid> h_pGrid;
    std::unique_ptr<DomainTransformer> h_pTrans;
    std::unique_ptr<MPMTimeIntegrator> h_pTimeIntegrator;
    std::vector<Model> h_models;
    std::vector<vector3T> h_vel;
    std::vector<unsigned int> h_indices;
};
