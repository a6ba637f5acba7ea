// Binning of caller-owned device positions with no device allocation.
//
// Some callers cannot allocate device memory on the call path: a host
// framework that owns and budgets every byte of device memory up front (an
// engine or a coupled solver that hands this library only views of its own
// buffers), or a latency-critical loop where cudaMalloc's implicit
// synchronisation and unpredictable cost are not allowed.  This entry point
// serves them: inputs and outputs are the caller's device buffers and all
// scratch lives in one file-scope __device__ array of fixed size, resolved once
// per device with cudaGetSymbolAddress.
//
// The array is shared by every call in the process: calls that overlap on the
// GPU (different streams, or host threads without ordering) race on it and
// must be serialised by the caller.  Its contents persist between calls, so
// everything that must start at zero is cleared on the call's stream first.
// The work is enqueued on the caller's stream, which must belong to the
// current device (the array resolved is the current device's).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "kernels.h"
#include "launch.cuh"
#include "scan.cuh"

namespace gmpm {

// Limits (also stated in include/gmpm.h).
constexpr int64_t kNoAllocMaxParticles = int64_t(1) << 20;   // 1,048,576
constexpr int kNoAllocMaxRes = 128;                          // nodes per axis -> page coordinates < 32
constexpr int kNoAllocKeyBits = 5;                           // bits per axis of the page key
constexpr uint32_t kNoAllocKeySpace = 1u << (3 * kNoAllocKeyBits);  // 32,768 pages: every page of the grid
constexpr int64_t kNoAllocCells = (int64_t)kNoAllocKeySpace * 64;

// Scratch layout (bytes, each region 256-byte aligned).
constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kOffCounters = 0;
constexpr size_t kOffKeys = align256(kOffCounters + sizeof(Counters));
constexpr size_t kOffPageFlag = align256(kOffKeys + kNoAllocMaxParticles * sizeof(uint32_t));
constexpr size_t kOffPageRank = align256(kOffPageFlag + kNoAllocKeySpace);
constexpr size_t kOffBlockKeys = align256(kOffPageRank + kNoAllocKeySpace * sizeof(int32_t));
constexpr size_t kOffCellCount = align256(kOffBlockKeys + kNoAllocKeySpace * sizeof(uint32_t));
constexpr size_t kOffCellStart = align256(kOffCellCount + kNoAllocCells * sizeof(int32_t));
constexpr size_t kOffScanTiles = align256(kOffCellStart + (kNoAllocCells + 1) * sizeof(int32_t));
constexpr size_t kScanTilesElems = (kNoAllocCells + kScanTile - 1) / kScanTile + 1;
constexpr size_t kNoAllocScratchBytes = align256(kOffScanTiles + kScanTilesElems * sizeof(int32_t));
static_assert(kNoAllocScratchBytes == GMPM_NOALLOC_SCRATCH_BYTES, "keep include/gmpm.h in step");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Kernel of bin.cu reused unchanged (the counting-sort passes go through the launchers of kernels.h).
__global__ void k_compact_keys(uint32_t key_space, const uint8_t* __restrict__ flag, const int32_t* __restrict__ rank,
                               uint32_t* __restrict__ out, int cap, Counters* cnt);

// Page/cell keys of interleaved xyz positions: the scene binning's cell_key
// (common.cuh; cal_cellId, Particle_kernal.cu:158-165).
__global__ void k_noalloc_keys(int64_t n, const float* __restrict__ pos, double inv_dx, int rx, int ry, int rz,
                               uint32_t* __restrict__ keys, uint8_t* __restrict__ page_flag, Counters* cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int res[3] = {rx, ry, rz};
    const float x[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    bool bad = false;
    const uint32_t key = cell_key(x, inv_dx, res, bad);
    if (bad) raise_flag(cnt, GMPM_FLAG_OUT_OF_DOMAIN);
    keys[i] = key;
    page_flag[key >> 6] = 1;
}

namespace {

// Device address of g_noalloc_scratch per device, resolved on first use.
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

cudaError_t scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = reinterpret_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace gmpm

extern "C" gmpm_status gmpm_bin_positions_noalloc(const float* positions, int64_t n, double dx, int res_x, int res_y,
                                                  int res_z, int32_t* perm, uint32_t* keys_sorted, uint32_t* flags,
                                                  void* stream) {
    using namespace gmpm;
    if (!positions || !perm || !keys_sorted || n <= 0 || !(dx > 0)) return GMPM_INVALID_ARG;
    if (n > kNoAllocMaxParticles) return GMPM_INVALID_ARG;
    const int res[3] = {res_x, res_y, res_z};
    for (int a = 0; a < 3; ++a)
        if (res[a] < 8 || res[a] > kNoAllocMaxRes) return GMPM_INVALID_ARG;
    unsigned char* base = nullptr;
    if (scratch_for_current_device(&base) != cudaSuccess) return GMPM_CUDA_ERROR;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    Counters* cnt = reinterpret_cast<Counters*>(base + kOffCounters);
    // n particles occupy at most n pages, so page ranks stay below min(n, key space):
    // only that many pages' cells are cleared and scanned
    const int32_t nb_cap = (int32_t)std::min<int64_t>(n, (int64_t)kNoAllocKeySpace);
    const int64_t ncell = (int64_t)nb_cap * 64;
    BinDev bin{};
    bin.n = n;
    bin.key_space = kNoAllocKeySpace;
    bin.nb_cap = nb_cap;
    bin.ng_cap = 0;
    bin.keys = reinterpret_cast<uint32_t*>(base + kOffKeys);
    bin.keys_sorted = keys_sorted;
    bin.perm = perm;
    bin.page_flag = base + kOffPageFlag;
    bin.page_rank = reinterpret_cast<int32_t*>(base + kOffPageRank);
    bin.block_keys = reinterpret_cast<uint32_t*>(base + kOffBlockKeys);
    bin.cell_count = reinterpret_cast<int32_t*>(base + kOffCellCount);
    bin.cell_start = reinterpret_cast<int32_t*>(base + kOffCellStart);
    ScanScratch scan{reinterpret_cast<int32_t*>(base + kOffScanTiles), (int64_t)kScanTilesElems};
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

    // state left by the previous call: clear what must start at zero
    if (e == cudaSuccess) e = cudaMemsetAsync(cnt, 0, sizeof(Counters), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bin.page_flag, 0, kNoAllocKeySpace, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bin.cell_count, 0, ncell * sizeof(int32_t), s);
    const int T = 256;
    const unsigned gn = (unsigned)((n + T - 1) / T);
    const unsigned gk = (kNoAllocKeySpace + T - 1) / T;
    if (e == cudaSuccess)
        e = launch_kernel(k_noalloc_keys, dim3(gn), dim3(T), 0, s, n, positions, 1.0 / dx, res_x, res_y, res_z,
                          bin.keys, bin.page_flag, cnt);
    if (e == cudaSuccess)
        e = scan_exclusive<uint8_t>(bin.page_flag, bin.page_rank, (int64_t)kNoAllocKeySpace, &cnt->n_blocks, scan, s);
    if (e == cudaSuccess)
        e = launch_kernel(k_compact_keys, dim3(gk), dim3(T), 0, s, kNoAllocKeySpace, (const uint8_t*)bin.page_flag,
                          (const int32_t*)bin.page_rank, bin.block_keys, (int)bin.nb_cap, cnt);
    if (e == cudaSuccess) e = launch_bin_hist(n, bin.keys, bin.page_rank, bin.cell_count, bin.nb_cap, s);
    if (e == cudaSuccess)
        e = scan_exclusive<int32_t>(bin.cell_count, bin.cell_start, ncell, bin.cell_start + ncell, scan, s,
                                    &cnt->n_blocks);
    if (e == cudaSuccess) e = cudaMemsetAsync(bin.cell_count, 0, ncell * sizeof(int32_t), s);
    if (e == cudaSuccess)
        e = launch_bin_scatter(n, bin.keys, bin.page_rank, bin.cell_start, bin.cell_count, perm, keys_sorted,
                               bin.nb_cap, s);
    if (e == cudaSuccess) e = launch_bin_canon(bin, cnt, sms, s);
    if (e == cudaSuccess && flags)
        e = cudaMemcpyAsync(flags, &cnt->flags, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? GMPM_OOM : GMPM_CUDA_ERROR;
    return GMPM_OK;
}
