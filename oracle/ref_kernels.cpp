// Known-answer driver for the reference's per-thread kernels.
//
// Test infrastructure only.  Built by oracle/Makefile (target `ref`): the
// kernel definitions come from oracle/_ref/ref_kernels.inc, which
// oracle/ref_extract.py takes at build time from the reference's own
// GPU_MPM/Particle_kernal.cu, TimeIntegrator.cu and ExplicitTimeIntegrator.cu.
// This file supplies what a CUDA compiler would: the qualifiers are defined
// away, blockIdx/threadIdx/blockDim are host variables, and launch() runs a
// grid serially, block by block and thread by thread.  That is exact for the
// kernels used here, which touch no shared memory, barriers, warp intrinsics or
// atomics.  The output goes to oracle/_ref/ref_kernels; tests/golden/
// make_golden.py runs it once to record fixtures.
//
// Host stand-ins for three device intrinsics:
//   __brevll  bit reversal of a 64-bit word (exact);
//   __clzll   count of leading zeros (exact; 64 for 0);
//   __fdividef single-precision divide.  The device intrinsic is an
//             approximate divide (within 2 ulp); here it is the correctly
//             rounded float quotient, so the recorded c = C/W of
//             undateGrid_kernal can differ from a GPU run of the reference in
//             the last float bits.
// Built without FMA contraction, so every product and sum rounds on its own.
//
// Modes (argv[1]); numbers are hex floats, one case per input line:
//   vonmises  in:  E nu dx V0 F0..F8 g alpha c psi_max   (F column-major,
//                  the reference's d_F planes)
//             out: VM F0..F8 g alpha psi_max FP contribution0..8 volume
//             Lamé constants from ElasticMaterial (Materials.cpp:4-13), then
//             applyVonMises (ExplicitTimeIntegrator.cu:132-370) and
//             computePhase_field_vol (:49-62) on its F.
//   grid      in:  first line "dt t bc" (bc 0: none, 1: collideWithGround,
//                  2: PullGrid_kernal); then one page per line: bx by bz and
//                  64 x 10 channel values (node-major, channels 0..9)
//             out: GRID v0 v1 v2 c per node (channels 1, 2, 3, 7)
//             undateGrid_kernal (TimeIntegrator.cu:63-111), then the chosen
//             boundary kernel (:117-165 or :169-261) with N = 256 (Setting.h).
//   cell      in:  one_over_dx x y z
//             out: CELL offset(hex) i j k — cal_cellId (Particle_kernal.cu:
//                  158-165) and calcIndex (TimeIntegrator.cu:53-61) of the
//                  particle as the first of its cell.
#include <math.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#define __host__
#define __device__
#define __global__
#define __forceinline__ inline

struct HostDim3 {
    unsigned x, y, z;
};
static HostDim3 threadIdx, blockIdx, blockDim, gridDim;
struct int3 {
    int x, y, z;
};

static inline unsigned long long __brevll(unsigned long long v) {
    unsigned long long r = 0;
    for (int b = 0; b < 64; ++b) r |= ((v >> b) & 1ull) << (63 - b);
    return r;
}
static inline int __clzll(long long v) { return v == 0 ? 64 : __builtin_clzll((unsigned long long)v); }
static inline float __fdividef(float a, float b) { return a / b; }

#include "Materials.h"
#include "QRSVD.hpp"
#include "SPGridMask.h"
#include "Setting.h"

#include "ref_kernels.inc"

template <class Kernel>
static void launch(unsigned blocks, unsigned threads, Kernel&& k) {
    gridDim = {blocks, 1, 1};
    blockDim = {threads, 1, 1};
    for (unsigned b = 0; b < blocks; ++b)
        for (unsigned t = 0; t < threads; ++t) {
            blockIdx = {b, 0, 0};
            threadIdx = {t, 0, 0};
            k();
        }
}

static bool read_values(char* line, std::vector<double>& v) {
    v.clear();
    for (char* tok = std::strtok(line, " \t\r\n"); tok; tok = std::strtok(nullptr, " \t\r\n"))
        v.push_back(std::strtod(tok, nullptr));
    return !v.empty();
}

static void put(double x) { std::printf(" %a", x); }

static int mode_vonmises() {
    std::vector<std::vector<double>> cases;
    std::vector<double> v;
    static char line[1 << 16];
    while (std::fgets(line, sizeof line, stdin))
        if (read_values(line, v)) {
            if (v.size() != 17) return 2;
            cases.push_back(v);
        }
    // one launch per case: each case brings its own material and dx
    for (const auto& c : cases) {
        ElasticMaterial mat(2, c[0], c[1], 1000.0, c[3]);
        const T dx = c[2], V0 = c[3];
        const int n = 1;
        T Fp[9], g = c[13], alpha = c[14], phase = c[15], psi = c[16], FP = 0, contrib[9], vol = 0;
        for (int q = 0; q < 9; ++q) Fp[q] = c[4 + q];
        launch(1, 1, [&] {
            applyVonMises(&g, &alpha, mat._lambda, mat._mu, dx, &FP, n, Fp, &psi, &phase, mat._kappa, V0, contrib);
        });
        launch(1, 1, [&] { computePhase_field_vol(n, Fp, V0, &vol); });
        std::printf("VM");
        for (int q = 0; q < 9; ++q) put(Fp[q]);
        put(g);
        put(alpha);
        put(psi);
        put(FP);
        for (int q = 0; q < 9; ++q) put(contrib[q]);
        put(vol);
        std::printf("\n");
    }
    return 0;
}

static int mode_grid() {
    static char line[1 << 20];
    std::vector<double> v;
    if (!std::fgets(line, sizeof line, stdin) || !read_values(line, v) || v.size() != 3) return 2;
    const T dt = v[0], t = v[1];
    const int bc = (int)v[2];
    SPGridMask sm(6, 3);
    sm.Cal_Masks();
    unsigned long long masks[3];
    sm.getMasks(masks);
    std::vector<unsigned long long> offsets;
    std::vector<std::vector<double>> pages;
    while (std::fgets(line, sizeof line, stdin))
        if (read_values(line, v)) {
            if (v.size() != 3 + 640) return 2;
            offsets.push_back(SPGridMask::Linear_Offset(masks, 4 * (int)v[0], 4 * (int)v[1], 4 * (int)v[2]));
            pages.push_back(v);
        }
    const size_t np = pages.size();
    const size_t per_page = MEMOFFSET / sizeof(T);  // 15 channels x 64 nodes
    std::vector<T> pool(np * per_page, 0.0);
    T* channels[15];
    for (int ch = 0; ch < 15; ++ch) channels[ch] = pool.data() + ch * 64;
    for (size_t p = 0; p < np; ++p)
        for (int node = 0; node < 64; ++node)
            for (int ch = 0; ch < 10; ++ch) pool[p * per_page + ch * 64 + node] = pages[p][3 + node * 10 + ch];
    launch((unsigned)np, 64, [&] { undateGrid_kernal(dt, channels); });
    if (bc == 1) launch((unsigned)np, 64, [&] { collideWithGround(masks, offsets.data(), channels); });
    if (bc == 2) launch((unsigned)np, 64, [&] { PullGrid_kernal(masks, offsets.data(), channels, t, dx); });
    for (size_t p = 0; p < np; ++p) {
        std::printf("GRID");
        for (int node = 0; node < 64; ++node)
            for (int ch : {1, 2, 3, 7}) put(pool[p * per_page + ch * 64 + node]);
        std::printf("\n");
    }
    return 0;
}

static int mode_cell() {
    SPGridMask sm(6, 3);
    sm.Cal_Masks();
    unsigned long long masks[3];
    sm.getMasks(masks);
    static char line[4096];
    std::vector<double> v;
    while (std::fgets(line, sizeof line, stdin))
        if (read_values(line, v)) {
            if (v.size() != 4) return 2;
            vector3T pos{v[1], v[2], v[3]};
            unsigned long long offset = 0;
            int first = 0;
            int3 node{0, 0, 0};
            launch(1, 1, [&] { cal_cellId(1, v[0], masks, &pos, &offset); });
            launch(1, 1, [&] { calcIndex(1, v[0], &first, &pos, &node); });
            std::printf("CELL %llx %d %d %d\n", offset, node.x, node.y, node.z);
        }
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_kernels vonmises|grid|cell < cases\n");
        return 2;
    }
    const std::string mode = argv[1];
    int rc = 2;
    if (mode == "vonmises") rc = mode_vonmises();
    if (mode == "grid") rc = mode_grid();
    if (mode == "cell") rc = mode_cell();
    if (rc) std::fprintf(stderr, "ref_kernels %s: bad input\n", argv[1]);
    return rc;
}
