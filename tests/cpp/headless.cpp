// Headless stand-in for the reference's GLUT driver (GPU_MPM/gl_main.cpp:477-508):
// MPMSimulator::build, then one simulateStick per frame, as display_func does
// (gl_main.cpp:304-314).  Writes the final positions in original particle
// order as raw float64 to argv[3].
//
//   headless <buildtype> <frames> <out.bin>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gmpm_simulator.hpp"

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: headless <buildtype> <frames> <out.bin>\n");
        return 2;
    }
    const unsigned buildtype = (unsigned)std::atoi(argv[1]);
    const int frames = std::atoi(argv[2]);
    MPMSimulator sim;
    if (!sim.build(buildtype)) {
        std::fprintf(stderr, "build failed\n");
        return 1;
    }
    float cfl = 0, pre = 0, simu = 0, pre_total = 0, simu_total = 0;
    try {
        for (int f = 0; f < frames; ++f) {
            sim.simulateStick(&cfl, &pre, &simu, 1);
            pre_total += pre;
            simu_total += simu;
        }
    } catch (const GmpmError& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    // positions in original order
    std::vector<double> pos(3 * (size_t)sim.numParticle);
    if (gmpm_read_particles(sim.scene(), GMPM_FIELD_POSITION, GMPM_DTYPE_F64, GMPM_ORDER_ORIGINAL, pos.data(),
                            pos.size() * sizeof(double), nullptr) != GMPM_OK)
        return 1;
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    std::fwrite(pos.data(), sizeof(double), pos.size(), f);
    std::fclose(f);
    std::printf("particles %u frames %d preprocess_ms %.3f simulation_ms %.3f h_pos[0] %.9f %.9f %.9f\n",
                sim.numParticle, frames, pre_total, simu_total, sim.h_pos[0].x, sim.h_pos[0].y, sim.h_pos[0].z);
    return 0;
}
