// Seeded synthetic scenes (host only).  Stand-ins for the reference's sampled
// assets (LoadSample.cpp:109-176); the SDF/OBJ inputs of its scenes are not
// shipped with the reference.
#include <cstdint>
#include <cstring>

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
