// Particle binning by SPGrid page/cell key, replacing the reference's hash +
// counting sort (Particles::sort_by_offsets, Particle_kernal.cu:158-249,484-542)
// and DomainTransformer::rebuild (Transformer_kernal.cu:15-209).
//
// Instead of an open-addressing page hash with unbounded probes and host
// syncs, pages are marked in a dense page-key table (the key space of the
// scene's grid), ranked by an exclusive scan (ascending page key = canonical
// page ids), and the +x/+y/+z neighbour pages are found by the same table.
// Particles are counting-sorted by (page rank, cell); the in-cell order is
// then made canonical (ascending previous slot), so the result equals a
// stable sort by (key, previous slot) bit for bit.  No host synchronisation.
#include <algorithm>
#include <cstdint>

#include "kernels.h"
#include "scan.cuh"

namespace gmpm {

// Particles per thread of the streaming binning kernels: each thread takes
// kBinILP particles one CTA width apart (coalesced per round) and issues all
// their loads before using any, so more requests are in flight per SM.
constexpr int kBinThreads = 256;
constexpr int kBinILP = 8;

// The kernels' bodies take the CTA's index within its scene's share of the
// launch (VB, common.cuh); the __global__ wrappers below each body serve a
// one-scene launch, the batched launches at the end of this file many scenes.

// The key pass: cell keys and page flags of positions that no G2P wrote
// (creation, restore, rebin).  A substep's binning starts from the keys its
// previous G2P formed for the positions it wrote.
template <typename R>
__device__ __forceinline__ void bin_keys_body(VB vb, int64_t n, const R* __restrict__ x0, const R* __restrict__ x1,
                                              const R* __restrict__ x2, const SceneDev<R>* __restrict__ sc,
                                              uint32_t* __restrict__ keys, uint8_t* __restrict__ page_flag,
                                              Counters* cnt) {
    const int64_t i0 = (int64_t)vb.b * kBinThreads * kBinILP + threadIdx.x;
    const double inv_dx = sc->inv_dx_d;
    const int res[3] = {sc->res[0], sc->res[1], sc->res[2]};
    R xs[kBinILP][3];
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) {
        const int64_t i = i0 + (int64_t)u * kBinThreads;
        if (i < n) {
            xs[u][0] = x0[i];
            xs[u][1] = x1[i];
            xs[u][2] = x2[i];
        }
    }
    bool bad = false;
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) {
        const int64_t i = i0 + (int64_t)u * kBinThreads;
        if (i >= n) continue;
        const uint32_t key = cell_key(xs[u], inv_dx, res, bad);
        keys[i] = key;
        page_flag[key >> 6] = 1;
    }
    if (bad) raise_flag(cnt, GMPM_FLAG_OUT_OF_DOMAIN);
}

template <typename R>
__global__ void __launch_bounds__(kBinThreads) k_bin_keys(int64_t n, const R* __restrict__ x0,
                                                          const R* __restrict__ x1, const R* __restrict__ x2,
                                                          const SceneDev<R>* __restrict__ sc,
                                                          uint32_t* __restrict__ keys,
                                                          uint8_t* __restrict__ page_flag, Counters* cnt) {
    bin_keys_body<R>(own_blocks(), n, x0, x1, x2, sc, keys, page_flag, cnt);
}

// Mark every active page and its 7 "+" neighbours as grid pages
// (supplementAdjacentPages, Transformer_kernal.cu:70-96).
__device__ __forceinline__ void mark_grid_body(VB vb, uint32_t key_space, const uint8_t* __restrict__ page_flag,
                                               uint8_t* __restrict__ grid_flag) {
    const uint32_t k = vb.b * blockDim.x + threadIdx.x;
    if (k >= key_space || !page_flag[k]) return;
    int bx, by, bz;
    page_coords(k, bx, by, bz);
#pragma unroll
    for (int d = 0; d < 8; ++d) grid_flag[page_key(bx + (d >> 2), by + ((d >> 1) & 1), bz + (d & 1))] = 1;
}

__global__ void k_mark_grid(uint32_t key_space, const uint8_t* __restrict__ page_flag, uint8_t* __restrict__ grid_flag) {
    mark_grid_body(own_blocks(), key_space, page_flag, grid_flag);
}

// Compact flagged keys into ascending order.
__device__ __forceinline__ void compact_keys_body(VB vb, uint32_t key_space, const uint8_t* __restrict__ flag,
                                                  const int32_t* __restrict__ rank, uint32_t* __restrict__ out,
                                                  int cap, Counters* cnt) {
    const uint32_t k = vb.b * blockDim.x + threadIdx.x;
    if (k >= key_space || !flag[k]) return;
    const int r = rank[k];
    if (r < cap)
        out[r] = k;
    else
        raise_flag(cnt, GMPM_FLAG_TABLE_OVERFLOW);
}

__global__ void k_compact_keys(uint32_t key_space, const uint8_t* __restrict__ flag, const int32_t* __restrict__ rank,
                               uint32_t* __restrict__ out, int cap, Counters* cnt) {
    compact_keys_body(own_blocks(), key_space, flag, rank, out, cap, cnt);
}

// Page topology: adj (establishPageTopology, Transformer_kernal.cu:98-114) and
// its inverse grid_src used by the fixed-order grid gather.
__device__ __forceinline__ void page_links_body(VB vb, const BinDev& bin, const Counters* cnt) {
    const int nb = min(cnt->n_blocks, bin.nb_cap);
    const int ng = min(cnt->n_grid_blocks, bin.ng_cap);
    const int t = vb.b * blockDim.x + threadIdx.x;
    const int slot = t & 7;
    const int idx = t >> 3;
    const int di = slot >> 2, dj = (slot >> 1) & 1, dk = slot & 1;
    if (idx < nb) {
        int bx, by, bz;
        page_coords(bin.block_keys[idx], bx, by, bz);
        const int r = bin.grid_rank[page_key(bx + di, by + dj, bz + dk)];
        bin.adj[idx * 8 + slot] = (r < bin.ng_cap) ? r : -1;  // overflow is flagged by k_compact_keys
    }
    if (idx < ng) {
        int gx, gy, gz;
        page_coords(bin.grid_keys[idx], gx, gy, gz);
        int src = -1;
        if (gx - di >= 0 && gy - dj >= 0 && gz - dk >= 0) {
            const uint32_t k = page_key(gx - di, gy - dj, gz - dk);
            if (k < bin.key_space && bin.page_flag[k]) {
                const int r = bin.page_rank[k];
                src = (r < bin.nb_cap) ? r : -1;
            }
        }
        bin.grid_src[idx * 8 + slot] = src;
    }
}

__global__ void k_page_links(BinDev bin, const Counters* cnt) { page_links_body(own_blocks(), bin, cnt); }

// Histogram of (page rank, cell) buckets with warp-aggregated atomics.
__device__ __forceinline__ void bin_hist_body(VB vb, int64_t n, const uint32_t* __restrict__ keys,
                                              const int32_t* __restrict__ page_rank, int32_t* __restrict__ cell_count,
                                              int nb_cap) {
    const int64_t i0 = (int64_t)vb.b * kBinThreads * kBinILP + threadIdx.x;
    uint32_t key[kBinILP];
    int rank[kBinILP];
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) key[u] = i0 + (int64_t)u * kBinThreads < n ? keys[i0 + (int64_t)u * kBinThreads] : 0u;
#pragma unroll
    for (int u = 0; u < kBinILP; ++u)
        rank[u] = i0 + (int64_t)u * kBinThreads < n ? page_rank[key[u] >> 6] : nb_cap;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) {
        const int bucket = rank[u] < nb_cap ? rank[u] * 64 + (int)(key[u] & 63) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, bucket);
        if (bucket >= 0 && lane == __ffs(peers) - 1) atomicAdd(&cell_count[bucket], __popc(peers));
    }
}

__global__ void __launch_bounds__(kBinThreads) k_bin_hist(int64_t n, const uint32_t* __restrict__ keys,
                                                          const int32_t* __restrict__ page_rank,
                                                          int32_t* __restrict__ cell_count, int nb_cap) {
    bin_hist_body(own_blocks(), n, keys, page_rank, cell_count, nb_cap);
}

// Scatter slots; lanes of one warp with the same bucket keep their order.
__device__ __forceinline__ void bin_scatter_body(VB vb, int64_t n, const uint32_t* __restrict__ keys,
                                                 const int32_t* __restrict__ page_rank,
                                                 const int32_t* __restrict__ cell_start, int32_t* __restrict__ fill,
                                                 int32_t* __restrict__ perm, uint32_t* __restrict__ keys_sorted,
                                                 int nb_cap) {
    const int64_t i0 = (int64_t)vb.b * kBinThreads * kBinILP + threadIdx.x;
    uint32_t key[kBinILP];
    int bucket[kBinILP], start[kBinILP];
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) key[u] = i0 + (int64_t)u * kBinThreads < n ? keys[i0 + (int64_t)u * kBinThreads] : 0u;
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) {
        const int r = i0 + (int64_t)u * kBinThreads < n ? page_rank[key[u] >> 6] : nb_cap;
        bucket[u] = r < nb_cap ? r * 64 + (int)(key[u] & 63) : -1;
    }
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) start[u] = bucket[u] >= 0 ? cell_start[bucket[u]] : 0;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int u = 0; u < kBinILP; ++u) {
        const unsigned peers = __match_any_sync(0xffffffffu, bucket[u]);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (bucket[u] >= 0 && lane == leader) base = atomicAdd(&fill[bucket[u]], __popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (bucket[u] >= 0) {
            const int slot = start[u] + base + __popc(peers & ((1u << lane) - 1u));
            perm[slot] = (int32_t)(i0 + (int64_t)u * kBinThreads);
            keys_sorted[slot] = key[u];
        }
    }
}

__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(int64_t n, const uint32_t* __restrict__ keys,
                                                             const int32_t* __restrict__ page_rank,
                                                             const int32_t* __restrict__ cell_start,
                                                             int32_t* __restrict__ fill, int32_t* __restrict__ perm,
                                                             uint32_t* __restrict__ keys_sorted, int nb_cap) {
    bin_scatter_body(own_blocks(), n, keys, page_rank, cell_start, fill, perm, keys_sorted, nb_cap);
}

// Canonical in-cell order: ascending previous slot.  Each warp takes one page
// (8 pages per CTA in flight, so the page's few dependent global round trips
// overlap across pages) and ranks every slot within its cell in shared memory
// (cells hold few particles).  A page above the warp's buffer is left to the
// whole CTA, which ranks it in windows of whole cells after the warps'
// pages; a single cell above the CTA buffer (thousands of particles in one
// cell, which only a failed state with clamped positions produces) keeps its
// scatter order and raises GMPM_FLAG_TABLE_OVERFLOW instead of being ranked
// in quadratic time.
constexpr int kCanonWarps = 8;
constexpr int kCanonWarpBuf = 768;
constexpr int kCanonBuf = kCanonWarps * kCanonWarpBuf;

// Rank slots [lo, hi) of a page (whole cells) by previous slot within their
// cells; buf holds perm[lo, hi).  Threads tid, tid + step, ... of the caller.
__device__ __forceinline__ void canon_rank(const BinDev& bin, const int32_t* cs, const int32_t* buf, int lo, int hi,
                                           int tid, int step) {
    for (int s = lo + tid; s < hi; s += step) {
        const int cell = (int)(bin.keys_sorted[s] & 63);
        const int a = cs[cell] - lo, e = cs[cell + 1] - lo;
        const int32_t v = buf[s - lo];
        int r = 0;
        for (int u = a; u < e; ++u) r += buf[u] < v;
        bin.perm[lo + a + r] = v;
    }
}

// Warp path: the scatter keeps the order of the lanes of one warp, so most
// cells already ascend by previous slot.  Only the cells with a descent are
// ranked; an ascending cell is its own canonical order.
__device__ __forceinline__ void canon_rank_warp(const BinDev& bin, const int32_t* cs, const int32_t* buf,
                                                uint8_t* bad, int lo, int hi, int lane) {
    for (int c = lane; c < 64; c += 32) bad[c] = 0;
    __syncwarp();
    for (int s = lo + lane; s < hi; s += 32) {
        const int cell = (int)(bin.keys_sorted[s] & 63);
        if (s > cs[cell] && buf[s - lo - 1] > buf[s - lo]) bad[cell] = 1;
    }
    __syncwarp();
    for (int s = lo + lane; s < hi; s += 32) {
        const int cell = (int)(bin.keys_sorted[s] & 63);
        if (!bad[cell]) continue;
        const int a = cs[cell] - lo, e = cs[cell + 1] - lo;
        const int32_t v = buf[s - lo];
        int r = 0;
        for (int u = a; u < e; ++u) r += buf[u] < v;
        bin.perm[lo + a + r] = v;
    }
}

__device__ __forceinline__ void bin_canon_body(VB vb, const BinDev& bin, Counters* cnt) {
    __shared__ int32_t buf[kCanonBuf];
    __shared__ int32_t cs[kCanonWarps][68];
    __shared__ uint8_t bad[kCanonWarps][64];
    __shared__ int big[kCanonWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nb = min(cnt->n_blocks, bin.nb_cap);
    int32_t* wbuf = buf + warp * kCanonWarpBuf;
    for (int g = vb.b * kCanonWarps; g < nb; g += vb.g * kCanonWarps) {
        const int b = g + warp;
        int is_big = 0;
        if (b < nb) {
            for (int q = lane; q < 65; q += 32) cs[warp][q] = bin.cell_start[(int64_t)b * 64 + q];
            __syncwarp();
            const int lo = cs[warp][0], hi = cs[warp][64];
            if (hi - lo <= kCanonWarpBuf) {
                for (int s = lo + lane; s < hi; s += 32) wbuf[s - lo] = bin.perm[s];
                __syncwarp();
                canon_rank_warp(bin, cs[warp], wbuf, bad[warp], lo, hi, lane);
            } else {
                is_big = 1;
            }
        }
        if (lane == 0) big[warp] = is_big;
        __syncthreads();
        // pages above a warp's buffer: the whole CTA, one at a time
        for (int w = 0; w < kCanonWarps; ++w) {
            if (!big[w]) continue;
            const int32_t* pcs = cs[w];
            int c0 = 0;
            while (c0 < 64) {
                int c1 = c0;
                while (c1 < 64 && pcs[c1 + 1] - pcs[c0] <= kCanonBuf) ++c1;
                if (c1 == c0) {
                    if (threadIdx.x == 0) raise_flag(cnt, GMPM_FLAG_TABLE_OVERFLOW);
                    c0 = c0 + 1;
                    continue;
                }
                const int lo = pcs[c0], hi = pcs[c1];
                for (int s = lo + (int)threadIdx.x; s < hi; s += blockDim.x) buf[s - lo] = bin.perm[s];
                __syncthreads();
                canon_rank(bin, pcs, buf, lo, hi, threadIdx.x, blockDim.x);
                __syncthreads();
                c0 = c1;
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(32 * kCanonWarps) k_bin_canon(BinDev bin, Counters* cnt) {
    bin_canon_body(own_blocks(), bin, cnt);
}

// ---------------------------------------------------------------------------

static unsigned bin_grid(int64_t n) {
    return (unsigned)std::max<int64_t>(1, (n + (int64_t)kBinThreads * kBinILP - 1) / ((int64_t)kBinThreads * kBinILP));
}

cudaError_t launch_bin_hist(int64_t n, const uint32_t* keys, const int32_t* page_rank, int32_t* cell_count, int nb_cap,
                            cudaStream_t s) {
    return launch_kernel(k_bin_hist, dim3(bin_grid(n)), dim3(kBinThreads), 0, s, n, keys, page_rank, cell_count,
                         nb_cap);
}

cudaError_t launch_bin_scatter(int64_t n, const uint32_t* keys, const int32_t* page_rank, const int32_t* cell_start,
                               int32_t* fill, int32_t* perm, uint32_t* keys_sorted, int nb_cap, cudaStream_t s) {
    return launch_kernel(k_bin_scatter, dim3(bin_grid(n)), dim3(kBinThreads), 0, s, n, keys, page_rank, cell_start,
                         fill, perm, keys_sorted, nb_cap);
}

cudaError_t launch_bin_canon(BinDev bin, Counters* cnt, int num_sms, cudaStream_t s) {
    return launch_kernel(k_bin_canon, dim3(num_sms * 8), dim3(32 * kCanonWarps), 0, s, bin, cnt);
}

template <typename R>
cudaError_t launch_binning(const SceneDev<R>* sc, const PState<R>& st, BinDev bin, ScanScratch scan, Counters* cnt,
                           int num_sms, cudaStream_t stream, bool keys_ready) {
    const int64_t n = bin.n;
    const int T = 256;
    const unsigned gn = bin_grid(n);
    const unsigned gk = (bin.key_space + T - 1) / T;
    cudaMemsetAsync(bin.grid_flag, 0, bin.key_space, stream);
    if (!keys_ready) {
        cudaMemsetAsync(bin.page_flag, 0, bin.key_space, stream);
        k_bin_keys<R><<<gn, kBinThreads, 0, stream>>>(n, st.x[0], st.x[1], st.x[2], sc, bin.keys, bin.page_flag, cnt);
    }
    scan_exclusive<uint8_t>(bin.page_flag, bin.page_rank, (int64_t)bin.key_space, &cnt->n_blocks, scan, stream);
    k_mark_grid<<<gk, T, 0, stream>>>(bin.key_space, bin.page_flag, bin.grid_flag);
    scan_exclusive<uint8_t>(bin.grid_flag, bin.grid_rank, (int64_t)bin.key_space, &cnt->n_grid_blocks, scan, stream);
    k_compact_keys<<<gk, T, 0, stream>>>(bin.key_space, bin.page_flag, bin.page_rank, bin.block_keys, bin.nb_cap, cnt);
    k_compact_keys<<<gk, T, 0, stream>>>(bin.key_space, bin.grid_flag, bin.grid_rank, bin.grid_keys, bin.ng_cap, cnt);
    const int links = max(bin.nb_cap, bin.ng_cap) * 8;
    k_page_links<<<(links + T - 1) / T, T, 0, stream>>>(bin, cnt);
    // the page flags' last use was the links: cleared for the G2P that keys the next positions
    if (keys_ready) cudaMemsetAsync(bin.page_flag, 0, bin.key_space, stream);
    const int64_t ncell = (int64_t)bin.nb_cap * 64;
    cudaMemsetAsync(bin.cell_count, 0, ncell * sizeof(int32_t), stream);
    launch_bin_hist(n, bin.keys, bin.page_rank, bin.cell_count, bin.nb_cap, stream);
    // the cells of the active pages only (the page scan above counted them)
    scan_exclusive<int32_t>(bin.cell_count, bin.cell_start, ncell, bin.cell_start + ncell, scan, stream,
                            &cnt->n_blocks);
    cudaMemsetAsync(bin.cell_count, 0, ncell * sizeof(int32_t), stream);
    launch_bin_scatter(n, bin.keys, bin.page_rank, bin.cell_start, bin.cell_count, bin.perm, bin.keys_sorted,
                       bin.nb_cap, stream);
    launch_bin_canon(bin, cnt, num_sms, stream);
    return cudaGetLastError();
}

template <typename R>
cudaError_t launch_keys(const SceneDev<R>* sc, const PState<R>& st, BinDev bin, Counters* cnt, cudaStream_t s) {
    k_bin_keys<R><<<bin_grid(bin.n), kBinThreads, 0, s>>>(bin.n, st.x[0], st.x[1], st.x[2], sc, bin.keys,
                                                                 bin.page_flag, cnt);
    return cudaGetLastError();
}
template cudaError_t launch_keys<float>(const SceneDev<float>*, const PState<float>&, BinDev, Counters*,
                                        cudaStream_t);
template cudaError_t launch_keys<double>(const SceneDev<double>*, const PState<double>&, BinDev, Counters*,
                                         cudaStream_t);

cudaError_t launch_mark_grid(BinDev bin, cudaStream_t s) {
    const int T = 256;
    k_mark_grid<<<(bin.key_space + T - 1) / T, T, 0, s>>>(bin.key_space, bin.page_flag, bin.grid_flag);
    return cudaGetLastError();
}

// ---- batched binning over many scenes ------------------------------------------

void batch_scene_ctas(int64_t n, uint32_t key_space, int nb_cap, int ng_cap, int sms, int real_bytes,
                      int ctas[kBatchMaps]) {
    auto cdiv = [](int64_t a, int64_t b) { return (int)std::max<int64_t>(1, (a + b - 1) / b); };
    const int64_t ncell = (int64_t)nb_cap * 64;
    ctas[BM_ZERO_FLAGS] = cdiv(key_space, 4096);
    ctas[BM_PARTICLES] = (int)bin_grid(n);
    ctas[BM_KEYSPACE] = cdiv(key_space, 256);
    ctas[BM_KEY_TILES] = cdiv(key_space, kScanTile);
    ctas[BM_LINKS] = cdiv((int64_t)std::max(nb_cap, ng_cap) * 8, 256);
    ctas[BM_ZERO_CELLS] = cdiv(ncell * 4, 4096);
    ctas[BM_CELL_TILES] = cdiv(ncell, kScanTile);
    ctas[BM_CANON] = std::max(1, std::min(cdiv(nb_cap, kCanonWarps), sms * 8));
    ctas[BM_P2G] = std::max(1, std::min(nb_cap, sms));
    ctas[BM_GRID] = std::max(1, std::min(ng_cap / 4 + 1, sms * 8));
    const int per_sm = real_bytes == 4 ? 2 : 1;  // G2P's resident CTAs per SM
    ctas[BM_G2P] = (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)sms * per_sm));
    ctas[BM_ONE] = 1;
}

// Zero `bytes` (a multiple of 4) from p in 4 KiB pieces: pieces vb.b, vb.b + vb.g, ...
__device__ __forceinline__ void zero_bytes_body(VB vb, void* p, int64_t bytes) {
    char* c = static_cast<char*>(p);
    const bool aligned = (reinterpret_cast<uintptr_t>(c) & 15) == 0;
    for (int64_t piece = (int64_t)vb.b * 4096; piece < bytes; piece += (int64_t)vb.g * 4096) {
        const int64_t off = piece + (int64_t)threadIdx.x * 16;
        if (off + 16 <= bytes && aligned) {
            *reinterpret_cast<uint4*>(c + off) = make_uint4(0u, 0u, 0u, 0u);
        } else {
            for (int q = 0; q < 16; q += 4)
                if (off + q + 4 <= bytes) *reinterpret_cast<uint32_t*>(c + off + q) = 0u;
        }
    }
}

// which: 1 grid flags; 2 cell counters; 3 cell counters and page flags (after
// the page flags' last use in the binning, for the G2P that sets them).
template <typename R>
__global__ void __launch_bounds__(256) k_batch_zero(const SceneArgs<R>* __restrict__ A, const int32_t* __restrict__ start,
                                                    int ns, int which) {
    VB vb;
    const BinDev& bin = A[scene_of_block(start, ns, vb)].bin;
    if (which == 1) zero_bytes_body(vb, bin.grid_flag, bin.key_space);
    if (which >= 2) zero_bytes_body(vb, bin.cell_count, (int64_t)bin.nb_cap * 64 * 4);
    if (which == 3) zero_bytes_body(vb, bin.page_flag, bin.key_space);
}

// The three scans of the binning: 0 page flags -> page ranks, 1 grid flags ->
// grid ranks, 2 cell counts -> cell starts.
template <int kWhich>
struct ScanSel;
template <>
struct ScanSel<0> {
    using T = uint8_t;
    static __device__ const T* in(const BinDev& b) { return b.page_flag; }
    static __device__ int64_t n(const BinDev& b) { return b.key_space; }
    static __device__ int32_t* out(const BinDev& b) { return b.page_rank; }
    static __device__ int32_t* total(const BinDev& b, Counters* c) { return &c->n_blocks; }
    static __device__ const int32_t* live(Counters*) { return nullptr; }
};
template <>
struct ScanSel<1> {
    using T = uint8_t;
    static __device__ const T* in(const BinDev& b) { return b.grid_flag; }
    static __device__ int64_t n(const BinDev& b) { return b.key_space; }
    static __device__ int32_t* out(const BinDev& b) { return b.grid_rank; }
    static __device__ int32_t* total(const BinDev& b, Counters* c) { return &c->n_grid_blocks; }
    static __device__ const int32_t* live(Counters*) { return nullptr; }
};
template <>
struct ScanSel<2> {
    using T = int32_t;
    static __device__ const T* in(const BinDev& b) { return b.cell_count; }
    static __device__ int64_t n(const BinDev& b) { return (int64_t)b.nb_cap * 64; }
    static __device__ int32_t* out(const BinDev& b) { return b.cell_start; }
    static __device__ int32_t* total(const BinDev& b, Counters*) { return b.cell_start + (int64_t)b.nb_cap * 64; }
    static __device__ const int32_t* live(Counters* c) { return &c->n_blocks; }  // the active pages' cells
};

template <typename R, int kWhich>
__global__ void __launch_bounds__(kScanThreads) k_batch_scan_reduce(const SceneArgs<R>* __restrict__ A,
                                                                    const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    using S = ScanSel<kWhich>;
    scan_reduce_body(vb, S::in(a.bin), S::n(a.bin), a.scan.tile_sums, S::live(a.cnt));
}

template <typename R, int kWhich>
__global__ void __launch_bounds__(kScanThreads) k_batch_scan_tiles(const SceneArgs<R>* __restrict__ A,
                                                                   const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    using S = ScanSel<kWhich>;
    const int64_t ntiles = (S::n(a.bin) + kScanTile - 1) / kScanTile;
    scan_tiles_body(a.scan.tile_sums, ntiles, S::total(a.bin, a.cnt));
}

template <typename R, int kWhich>
__global__ void __launch_bounds__(kScanThreads) k_batch_scan_apply(const SceneArgs<R>* __restrict__ A,
                                                                   const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    using S = ScanSel<kWhich>;
    scan_apply_body(vb, S::in(a.bin), S::n(a.bin), a.scan.tile_sums, S::out(a.bin), S::live(a.cnt));
}

template <typename R>
__global__ void __launch_bounds__(256) k_batch_mark(const SceneArgs<R>* __restrict__ A,
                                                    const int32_t* __restrict__ start, int ns) {
    VB vb;
    const BinDev& bin = A[scene_of_block(start, ns, vb)].bin;
    mark_grid_body(vb, bin.key_space, bin.page_flag, bin.grid_flag);
}

template <typename R>
__global__ void __launch_bounds__(256) k_batch_compact(const SceneArgs<R>* __restrict__ A,
                                                       const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    compact_keys_body(vb, a.bin.key_space, a.bin.page_flag, a.bin.page_rank, a.bin.block_keys, a.bin.nb_cap, a.cnt);
    compact_keys_body(vb, a.bin.key_space, a.bin.grid_flag, a.bin.grid_rank, a.bin.grid_keys, a.bin.ng_cap, a.cnt);
}

template <typename R>
__global__ void __launch_bounds__(256) k_batch_links(const SceneArgs<R>* __restrict__ A,
                                                     const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    page_links_body(vb, a.bin, a.cnt);
}

template <typename R>
__global__ void __launch_bounds__(kBinThreads) k_batch_hist(const SceneArgs<R>* __restrict__ A,
                                                            const int32_t* __restrict__ start, int ns) {
    VB vb;
    const BinDev& bin = A[scene_of_block(start, ns, vb)].bin;
    bin_hist_body(vb, bin.n, bin.keys, bin.page_rank, bin.cell_count, bin.nb_cap);
}

template <typename R>
__global__ void __launch_bounds__(kBinThreads) k_batch_scatter(const SceneArgs<R>* __restrict__ A,
                                                               const int32_t* __restrict__ start, int ns) {
    VB vb;
    const BinDev& bin = A[scene_of_block(start, ns, vb)].bin;
    bin_scatter_body(vb, bin.n, bin.keys, bin.page_rank, bin.cell_start, bin.cell_count, bin.perm, bin.keys_sorted,
                     bin.nb_cap);
}

template <typename R>
__global__ void __launch_bounds__(32 * kCanonWarps) k_batch_canon(const SceneArgs<R>* __restrict__ A,
                                                                  const int32_t* __restrict__ start, int ns) {
    VB vb;
    const SceneArgs<R>& a = A[scene_of_block(start, ns, vb)];
    bin_canon_body(vb, a.bin, a.cnt);
}

// The binning of every scene of a batch: the same steps as launch_binning with
// keys_ready, each one launch over all scenes.
template <typename R>
cudaError_t launch_batch_binning(const SceneArgs<R>* A, const BatchPlan& P, cudaStream_t s) {
    const int ns = P.n_scenes;
    auto T = [&](int m) { return dim3((unsigned)P.total[m]); };
    auto S = [&](int m) { return P.start[m]; };
    cudaError_t e = launch_kernel(k_batch_zero<R>, T(BM_ZERO_FLAGS), dim3(256), 0, s, A, S(BM_ZERO_FLAGS), ns, 1);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_reduce<R, 0>, T(BM_KEY_TILES), dim3(kScanThreads), 0, s, A, S(BM_KEY_TILES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_tiles<R, 0>, T(BM_ONE), dim3(kScanThreads), 0, s, A, S(BM_ONE), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_apply<R, 0>, T(BM_KEY_TILES), dim3(kScanThreads), 0, s, A, S(BM_KEY_TILES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_mark<R>, T(BM_KEYSPACE), dim3(256), 0, s, A, S(BM_KEYSPACE), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_reduce<R, 1>, T(BM_KEY_TILES), dim3(kScanThreads), 0, s, A, S(BM_KEY_TILES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_tiles<R, 1>, T(BM_ONE), dim3(kScanThreads), 0, s, A, S(BM_ONE), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_apply<R, 1>, T(BM_KEY_TILES), dim3(kScanThreads), 0, s, A, S(BM_KEY_TILES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_compact<R>, T(BM_KEYSPACE), dim3(256), 0, s, A, S(BM_KEYSPACE), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_links<R>, T(BM_LINKS), dim3(256), 0, s, A, S(BM_LINKS), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_zero<R>, T(BM_ZERO_CELLS), dim3(256), 0, s, A, S(BM_ZERO_CELLS), ns, 3);
    if (e == cudaSuccess) e = launch_kernel(k_batch_hist<R>, T(BM_PARTICLES), dim3(kBinThreads), 0, s, A, S(BM_PARTICLES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_reduce<R, 2>, T(BM_CELL_TILES), dim3(kScanThreads), 0, s, A, S(BM_CELL_TILES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_tiles<R, 2>, T(BM_ONE), dim3(kScanThreads), 0, s, A, S(BM_ONE), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scan_apply<R, 2>, T(BM_CELL_TILES), dim3(kScanThreads), 0, s, A, S(BM_CELL_TILES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_zero<R>, T(BM_ZERO_CELLS), dim3(256), 0, s, A, S(BM_ZERO_CELLS), ns, 2);
    if (e == cudaSuccess) e = launch_kernel(k_batch_scatter<R>, T(BM_PARTICLES), dim3(kBinThreads), 0, s, A, S(BM_PARTICLES), ns);
    if (e == cudaSuccess) e = launch_kernel(k_batch_canon<R>, T(BM_CANON), dim3(32 * kCanonWarps), 0, s, A, S(BM_CANON), ns);
    return e;
}
template cudaError_t launch_batch_binning<float>(const SceneArgs<float>*, const BatchPlan&, cudaStream_t);
template cudaError_t launch_batch_binning<double>(const SceneArgs<double>*, const BatchPlan&, cudaStream_t);

template cudaError_t launch_binning<float>(const SceneDev<float>*, const PState<float>&, BinDev, ScanScratch,
                                           Counters*, int, cudaStream_t, bool);
template cudaError_t launch_binning<double>(const SceneDev<double>*, const PState<double>&, BinDev, ScanScratch,
                                            Counters*, int, cudaStream_t, bool);

}  // namespace gmpm
