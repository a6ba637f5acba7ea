// Device-wide exclusive prefix sum (reduce -> scan tile sums -> apply), used
// for page ranks and cell offsets.  Replaces the reference's recursive block
// scan and Thrust scans (cuda_kernal_tools.cu:15-203, Transformer_kernal.cu:142-207).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"
#include "launch.cuh"

namespace gmpm {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

struct ScanScratch {
    int32_t* tile_sums;  // capacity: ceil(max_n / kScanTile) + 1
    int64_t capacity;
};

template <typename TIn>
__device__ __forceinline__ void scan_load(const TIn* in, int64_t n, int64_t base, int32_t v[kScanItems]) {
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        const int64_t idx = base + q;
        v[q] = (idx < n) ? (int32_t)in[idx] : 0;
    }
}

__device__ __forceinline__ int32_t block_exclusive_sum(int32_t x, int32_t* total) {
    __shared__ int32_t warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int32_t w = (lane < kScanThreads / 32) ? warp_sums[lane] : 0;
        int32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kScanThreads / 32) warp_sums[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1) *total = wi;
    }
    __syncthreads();
    const int32_t r = warp_sums[warp] + incl - x;
    __syncthreads();
    return r;
}

// Entries scanned: all n, or with `live` (a device count of live blocks of 64
// entries, the active pages of a cell scan, whose capacity is larger) only the
// live entries.  The scan then writes the live entries and the one after them,
// which receives the total; the entries beyond are left as they are, and no
// reader looks past the live pages.
__device__ __forceinline__ int64_t scan_live_len(int64_t n, const int32_t* live) {
    return live ? min(n, (int64_t)max(*live, 0) * 64) : n;
}

// Bodies take the CTA's tile index within its scene's scan (VB, common.cuh),
// so that the same code serves one-scene and batched launches.
template <typename TIn>
__device__ __forceinline__ void scan_reduce_body(VB vb, const TIn* __restrict__ in, int64_t n,
                                                 int32_t* __restrict__ tile_sums, const int32_t* live = nullptr) {
    const int64_t m = scan_live_len(n, live);
    if ((int64_t)vb.b * kScanTile >= m) {  // a tile past the live entries (whole CTA)
        if (threadIdx.x == 0) tile_sums[vb.b] = 0;
        return;
    }
    const int64_t base = (int64_t)vb.b * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    scan_load(in, m, base, v);
    int32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) s += v[q];
    __shared__ int32_t tot;
    block_exclusive_sum(s, &tot);
    if (threadIdx.x == 0) tile_sums[vb.b] = tot;
}

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const TIn* __restrict__ in, int64_t n,
                                                               int32_t* __restrict__ tile_sums,
                                                               const int32_t* __restrict__ live) {
    scan_reduce_body(own_blocks(), in, n, tile_sums, live);
}

// Single CTA: exclusive scan of the tile sums in place, total to *total.
__device__ __forceinline__ void scan_tiles_body(int32_t* __restrict__ tile_sums, int64_t ntiles,
                                                int32_t* __restrict__ total) {
    __shared__ int32_t chunk_total;
    int32_t carry = 0;
    for (int64_t base = 0; base < ntiles; base += kScanTile) {
        const int64_t b = base + (int64_t)threadIdx.x * kScanItems;
        int32_t v[kScanItems];
        scan_load(tile_sums, ntiles, b, v);
        int32_t s = 0;
#pragma unroll
        for (int q = 0; q < kScanItems; ++q) s += v[q];
        int32_t run = block_exclusive_sum(s, &chunk_total) + carry;
#pragma unroll
        for (int q = 0; q < kScanItems; ++q) {
            if (b + q < ntiles) tile_sums[b + q] = run;
            run += v[q];
        }
        carry += chunk_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

static __global__ void __launch_bounds__(kScanThreads) k_scan_tiles(int32_t* __restrict__ tile_sums, int64_t ntiles,
                                                              int32_t* __restrict__ total) {
    scan_tiles_body(tile_sums, ntiles, total);
}

template <typename TIn>
__device__ __forceinline__ void scan_apply_body(VB vb, const TIn* __restrict__ in, int64_t n,
                                                const int32_t* __restrict__ tile_offsets, int32_t* __restrict__ out,
                                                const int32_t* live = nullptr) {
    const int64_t m = scan_live_len(n, live);
    const int64_t w = min(n, m + 1);  // entries written: the live ones and the total after them
    if ((int64_t)vb.b * kScanTile >= w) return;  // whole CTA
    const int64_t base = (int64_t)vb.b * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    scan_load(in, m, base, v);
    int32_t s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) s += v[q];
    __shared__ int32_t tot;
    int32_t run = block_exclusive_sum(s, &tot) + tile_offsets[vb.b];
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (base + q < w) out[base + q] = run;
        run += v[q];
    }
}

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const TIn* __restrict__ in, int64_t n,
                                                              const int32_t* __restrict__ tile_offsets,
                                                              int32_t* __restrict__ out,
                                                              const int32_t* __restrict__ live) {
    scan_apply_body(own_blocks(), in, n, tile_offsets, out, live);
}

// out[i] = sum_{j<i} in[j] for i < n; *total = sum of all.  With `live` (see
// scan_live_len) only the live entries are read and the live entries and the
// one after them written.  Returns the status of its own launches.
template <typename TIn>
inline cudaError_t scan_exclusive(const TIn* in, int32_t* out, int64_t n, int32_t* total, ScanScratch s,
                                  cudaStream_t stream, const int32_t* live = nullptr) {
    const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
    cudaError_t e = launch_kernel(k_scan_reduce<TIn>, dim3((unsigned)ntiles), dim3(kScanThreads), 0, stream, in, n,
                                  s.tile_sums, live);
    if (e == cudaSuccess) e = launch_kernel(k_scan_tiles, dim3(1), dim3(kScanThreads), 0, stream, s.tile_sums, ntiles, total);
    if (e == cudaSuccess)
        e = launch_kernel(k_scan_apply<TIn>, dim3((unsigned)ntiles), dim3(kScanThreads), 0, stream, in, n,
                          (const int32_t*)s.tile_sums, out, live);
    return e;
}

inline int64_t scan_scratch_elems(int64_t max_n) { return (max_n + kScanTile - 1) / kScanTile + 1; }

}  // namespace gmpm
