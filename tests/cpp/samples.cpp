// The facade's Sample class (include/gmpm_simulator.hpp), used as the
// reference's Simulator.cpp uses its Sample: prints each sampler's particles
// as "%a %a %a" lines after a "COUNT n" line.
//
//   samples obj <path> | cube <N> | sdf <path> cx cy cz rx ry rz
#include <cstdio>
#include <cstdlib>
#include <string>

#include "gmpm_simulator.hpp"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    const std::string mode = argv[1];
    std::vector<vector3T> pts;
    try {
        if (mode == "obj") {
            pts = Sample().readObj(argv[2]);
        } else if (mode == "cube") {
            pts = Sample((unsigned)std::atoi(argv[2])).Initialize_Data_cube();
        } else if (mode == "sdf" && argc >= 9) {
            unsigned center[3], res[3];
            for (int a = 0; a < 3; ++a) {
                center[a] = (unsigned)std::atoi(argv[3 + a]);
                res[a] = (unsigned)std::atoi(argv[6 + a]);
            }
            pts = Sample().Initial_data(center, res, argv[2]);
        } else {
            return 2;
        }
    } catch (const GmpmError& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    std::printf("COUNT %zu\n", pts.size());
    for (const vector3T& q : pts) std::printf("%a %a %a\n", q.x, q.y, q.z);
    return 0;
}
