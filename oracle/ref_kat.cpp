// Known-answer driver for the reference's host-compilable code.
//
// Test infrastructure only. Built by oracle/Makefile (target `ref`) from the
// reference's own sources where they lie (GPU_MPM/SPGridMask.cpp,
// GPU_MPM/Materials.cpp and the header-only SVD GPU_MPM/QRSVD.hpp +
// GPU_MPM/givens.hpp, the latter against the container shim in
// oracle/eigen_shim). Output goes to oracle/_ref/ref_kat. Nothing here is part
// of the product; tests/golden/make_golden.py runs it once to record fixtures.
//
// Modes (argv[1]):
//   masks                 print the three SPGrid masks (SPGridMask.cpp:119-129)
//   offsets               read "i j k" lines, print Linear_Offset (SPGridMask.cpp:84-87)
//   svd                   read 9 hex-float entries per line (row-major F),
//                         print U (row-major), S, V (row-major) from
//                         __GEIGEN__::math::msvd (QRSVD.hpp:327-374)
//   material              read "E nu rho vol" lines, print lambda mu kappa M
//                         (Materials.cpp:4-13)
//   obj PATH              Sample::readObj (LoadSample.cpp:163-176) of PATH
//   cube                  Sample::Initialize_Data_cube (LoadSample.cpp:179-213)
//   sdf PATH cx cy cz rx ry rz
//                         Sample::Initial_data (LoadSample.cpp:109-161) of the
//                         SDF at PATH, with the C library generator in its
//                         initial state, as in the reference's run
// The sampling modes print the particle count, then one "%a %a %a" line per
// particle.
#include <math.h>  // brings the double overloads of abs() into the global namespace
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#define __host__
#define __device__
#include "QRSVD.hpp"
#include "SPGridMask.h"
#include "Materials.h"
#include "LoadSample.h"

static void print_hex(double v) { std::printf("%a", v); }

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_kat masks|offsets|svd|material|obj|cube|sdf\n");
        return 2;
    }
    std::string mode = argv[1];
    if (mode == "masks") {
        // SPGridMask(Log2(sizeof(CH_STRUCT)), Log2(sizeof(T))) — the constructor
        // ignores its arguments and fixes struct_size=6, element_size=2.
        SPGridMask m(6, 3);
        m.Cal_Masks();  // also prints the bitsets to stdout
        unsigned long long mk[3];
        m.getMasks(mk);
        std::printf("MASKS %llx %llx %llx\n", mk[0], mk[1], mk[2]);
        return 0;
    }
    if (mode == "offsets") {
        SPGridMask m(6, 3);
        m.Cal_Masks();
        unsigned long long mk[3];
        m.getMasks(mk);
        int i, j, k;
        while (std::scanf("%d %d %d", &i, &j, &k) == 3)
            std::printf("OFFSET %d %d %d %llx\n", i, j, k, SPGridMask::Linear_Offset(mk, i, j, k));
        return 0;
    }
    if (mode == "svd") {
        double a[9];
        char buf[64];
        for (;;) {
            bool ok = true;
            for (int q = 0; q < 9; ++q) {
                if (std::scanf("%63s", buf) != 1) { ok = false; break; }
                a[q] = std::strtod(buf, nullptr);
            }
            if (!ok) break;
            double u[9], v[9], s[3];
            __GEIGEN__::math::msvd(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8],
                                   u[0], u[1], u[2], u[3], u[4], u[5], u[6], u[7], u[8],
                                   s[0], s[1], s[2],
                                   v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8]);
            std::printf("SVD");
            for (int q = 0; q < 9; ++q) { std::printf(" "); print_hex(u[q]); }
            for (int q = 0; q < 3; ++q) { std::printf(" "); print_hex(s[q]); }
            for (int q = 0; q < 9; ++q) { std::printf(" "); print_hex(v[q]); }
            std::printf("\n");
        }
        return 0;
    }
    if (mode == "material") {
        double E, nu, rho, vol;
        while (std::scanf("%lf %lf %lf %lf", &E, &nu, &rho, &vol) == 4) {
            ElasticMaterial m(2, E, nu, rho, vol);
            std::printf("MATERIAL ");
            print_hex(m._lambda); std::printf(" ");
            print_hex(m._mu); std::printf(" ");
            print_hex(m._kappa); std::printf(" ");
            print_hex(m.parabolic_M); std::printf("\n");
        }
        return 0;
    }
    if (mode == "obj" || mode == "cube" || mode == "sdf") {
        Sample sample;
        std::vector<vector3T> pts;
        if (mode == "obj" && argc >= 3) {
            pts = sample.readObj(argv[2]);
        } else if (mode == "cube") {
            pts = sample.Initialize_Data_cube();
        } else if (mode == "sdf" && argc >= 9) {
            unsigned int center[3], res[3];
            for (int a = 0; a < 3; ++a) {
                center[a] = (unsigned)std::atoi(argv[3 + a]);
                res[a] = (unsigned)std::atoi(argv[6 + a]);
            }
            pts = sample.Initial_data(center, res, argv[2]);
        } else {
            std::fprintf(stderr, "bad arguments for %s\n", argv[1]);
            return 2;
        }
        std::fflush(stdout);
        std::printf("COUNT %zu\n", pts.size());
        for (const vector3T& q : pts) {
            print_hex(q.x); std::printf(" ");
            print_hex(q.y); std::printf(" ");
            print_hex(q.z); std::printf("\n");
        }
        return 0;
    }
    std::fprintf(stderr, "unknown mode %s\n", argv[1]);
    return 2;
}
