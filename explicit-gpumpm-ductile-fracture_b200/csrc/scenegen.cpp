// Seeded synthetic scenes (host only).  Stand-ins for the reference's sampled
// assets (LoadSample.cpp:109-176); the SDF/OBJ inputs of its scenes are not
// shipped with the reference.  Also the reference's own samplers (readObj,
// Initialize_Data_cube, Initial_data), restated to produce the same particles.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <vector>

#include "gmpm.h"

namespace {

struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

bool in_notch(const gmpm_scene_geometry& g, int iy, int iz) {
    if (g.kind != 0 || g.notch_width <= 0 || g.notch_depth <= 0) return false;
    const int z0 = g.cells[2] / 2 - g.notch_width / 2;
    return iz >= z0 && iz < z0 + g.notch_width && iy < g.notch_depth;
}

}  // namespace

extern "C" gmpm_status gmpm_generate_particles(const gmpm_scene_geometry* g, int64_t* count, double* positions,
                                               int32_t* material_ids, int64_t capacity) {
    if (!g || !count) return GMPM_INVALID_ARG;
    if (g->kind < 0 || g->kind > 2 || g->ppc <= 0 || !(g->dx > 0)) return GMPM_INVALID_ARG;
    for (int a = 0; a < 3; ++a)
        if (g->cells[a] <= 0) return GMPM_INVALID_ARG;
    const int plates = (g->kind == 1) ? g->n_plates : 1;
    if (plates <= 0 || plates > GMPM_MAX_MATERIALS || g->gap_cells < 0) return GMPM_INVALID_ARG;
    int64_t total = 0;
    for (int ix = 0; ix < g->cells[0]; ++ix)
        for (int iy = 0; iy < g->cells[1]; ++iy)
            for (int iz = 0; iz < g->cells[2]; ++iz)
                if (!in_notch(*g, iy, iz)) total += g->ppc;
    total *= plates;
    *count = total;
    if (!positions) return GMPM_OK;
    if (capacity < total) return GMPM_INVALID_ARG;
    SplitMix64 rng{g->seed};
    int64_t p = 0;
    for (int k = 0; k < plates; ++k) {
        const int yoff = k * (g->cells[1] + g->gap_cells);
        for (int ix = 0; ix < g->cells[0]; ++ix)
            for (int iy = 0; iy < g->cells[1]; ++iy)
                for (int iz = 0; iz < g->cells[2]; ++iz) {
                    if (in_notch(*g, iy, iz)) continue;
                    for (int q = 0; q < g->ppc; ++q) {
                        const int cell[3] = {ix, iy + yoff, iz};
                        for (int a = 0; a < 3; ++a) {
                            const double x = g->origin[a] + ((double)cell[a] + rng.uniform()) * g->dx;
                            positions[3 * p + a] = (double)(float)x;
                        }
                        if (material_ids) material_ids[p] = k;
                        ++p;
                    }
                }
    }
    return GMPM_OK;
}

// ---- the reference's samplers ----------------------------------------------

namespace {

gmpm_status emit(const std::vector<double>& xyz, int64_t* count, double* positions, int64_t capacity) {
    const int64_t n = (int64_t)(xyz.size() / 3);
    *count = n;
    if (!positions) return GMPM_OK;
    if (capacity < n) return GMPM_INVALID_ARG;
    std::memcpy(positions, xyz.data(), xyz.size() * sizeof(double));
    return GMPM_OK;
}

// Level set of an SDF file (LoadSDF): values at (i, j, k), i fastest.
struct LevelSet {
    int ni = 0, nj = 0, nk = 0;
    std::vector<double> phi;
    double at(int i, int j, int k) const { return phi[(size_t)i + (size_t)ni * ((size_t)j + (size_t)nj * k)]; }
    // fetchGridTrilinear (LoadSample.cpp:40-62): corners by floor and ceil of
    // each coordinate, blended along x, then y, then z
    double trilinear(double x, double y, double z) const {
        const double fx = x - std::floor(x), fy = y - std::floor(y), fz = z - std::floor(z);
        const int x0 = (int)std::floor(x), x1 = (int)std::ceil(x);
        const int y0 = (int)std::floor(y), y1 = (int)std::ceil(y);
        const int z0 = (int)std::floor(z), z1 = (int)std::ceil(z);
        const double c00 = at(x0, y0, z0) * (1 - fx) + at(x1, y0, z0) * fx;
        const double c01 = at(x0, y0, z1) * (1 - fx) + at(x1, y0, z1) * fx;
        const double c10 = at(x0, y1, z0) * (1 - fx) + at(x1, y1, z0) * fx;
        const double c11 = at(x0, y1, z1) * (1 - fx) + at(x1, y1, z1) * fx;
        const double c0 = c00 * (1 - fy) + c10 * fy;
        const double c1 = c01 * (1 - fy) + c11 * fy;
        return c0 * (1 - fz) + c1 * fz;
    }
};

}  // namespace

extern "C" gmpm_status gmpm_sample_obj(const char* path, int64_t* count, double* positions, int64_t capacity) {
    if (!path || !count) return GMPM_INVALID_ARG;
    std::ifstream in(path);
    if (!in) return GMPM_IO_ERROR;
    std::vector<double> xyz;
    char tag;
    double x, y, z;
    while (in >> tag >> x >> y >> z) {
        xyz.push_back(x);
        xyz.push_back(y - (double)0.2f);
        xyz.push_back(z);
    }
    return emit(xyz, count, positions, capacity);
}

extern "C" gmpm_status gmpm_sample_cube(int32_t n_grid, int64_t* count, double* positions, int64_t capacity) {
    if (!count || n_grid < 8) return GMPM_INVALID_ARG;
    const int N = n_grid;
    const double dx = 1.0 / N;
    const int x0 = N / 2 - N / 20, x1 = N / 2 + N / 20;
    const int z0 = N / 2 - N / 8, z1 = N / 2 + N / 8;
    const double ddx = dx / 3;  // lattice spacing: dx / (2 * 1 + 1)
    std::vector<double> xyz;
    xyz.reserve((size_t)(x1 - x0) * (x1 - x0) * (z1 - z0) * 81);
    for (int i = x0; i < x1; ++i)
        for (int j = x0; j < x1; ++j)
            for (int k = z0; k < z1; ++k) {
                const double c[3] = {(i + 0.5) * dx, (j + 0.5) * dx, (k + 0.5) * dx};
                for (int a = -1; a <= 1; ++a)
                    for (int b = -1; b <= 1; ++b)
                        for (int d = -1; d <= 1; ++d) {
                            xyz.push_back(c[0] + a * ddx);
                            xyz.push_back(c[1] + b * ddx);
                            xyz.push_back(c[2] + d * ddx);
                        }
            }
    return emit(xyz, count, positions, capacity);
}

extern "C" gmpm_status gmpm_sample_sdf(const char* path, const uint32_t center[3], const uint32_t res[3], double dx,
                                       uint32_t seed, int64_t* count, double* positions, int64_t capacity) {
    if (!path || !center || !res || !count || !(dx > 0)) return GMPM_INVALID_ARG;
    std::ifstream in(path);
    if (!in) return GMPM_IO_ERROR;
    LevelSet ls;
    double box[3], ldx;
    if (!(in >> ls.ni >> ls.nj >> ls.nk >> box[0] >> box[1] >> box[2] >> ldx)) return GMPM_IO_ERROR;
    if (ls.ni < 4 || ls.nj < 4 || ls.nk < 4) return GMPM_IO_ERROR;
    ls.phi.resize((size_t)ls.ni * ls.nj * ls.nk);
    for (double& v : ls.phi)
        if (!(in >> v)) return GMPM_IO_ERROR;

    // placement (Initial_data): the level set's cells 1 .. n-2 scaled into
    // res[] grid cells from the corner (center - res/2, center_y + res_y/4, ...)
    int corner[3];
    for (int a = 0; a < 3; ++a) corner[a] = (int)(center[a] - .5 * res[a]);
    corner[1] = (int)(center[1] + 0.25 * res[1]);
    const int lo = 1;
    const int hi[3] = {ls.ni - 2, ls.nj - 2, ls.nk - 2};
    double scale = 0.0;
    for (int a = 0; a < 3; ++a) {
        // the reference computes each axis scale in single precision
        const double sa = (double)(1.f * (int)res[a] / (hi[a] - lo));
        scale = a == 0 ? sa : (sa < scale ? sa : scale);
    }
    const double per_cell = 20 * scale * scale * scale;

    // GenerateUniformSamples (LoadSample.cpp:64-105): cells with a negative
    // corner, then rejection samples over the whole level-set box
    int cells = 0;
    for (int i = 0; i < ls.ni - 1; ++i)
        for (int j = 0; j < ls.nj - 1; ++j)
            for (int k = 0; k < ls.nk - 1; ++k) {
                bool inside = false;
                for (int c = 0; c < 8 && !inside; ++c) inside = ls.at(i + (c >> 2), j + ((c >> 1) & 1), k + (c & 1)) < 0;
                cells += inside ? 1 : 0;
            }
    const int n = (int)(cells * per_cell);
    std::vector<double> xyz;
    xyz.reserve((size_t)n * 3);
    std::srand(seed);
    for (int s = 0; s < n; ++s) {
        double p[3];
        do {
            p[0] = (double)std::rand() / RAND_MAX * (ls.ni - 1);
            p[1] = (double)std::rand() / RAND_MAX * (ls.nj - 1);
            p[2] = (double)std::rand() / RAND_MAX * (ls.nk - 1);
        } while (ls.trilinear(p[0], p[1], p[2]) >= 0);
        for (int a = 0; a < 3; ++a) xyz.push_back(((p[a] - lo) * scale + corner[a] + 4) * dx);
    }
    return emit(xyz, count, positions, capacity);
}
