// Asynchronous global -> shared copies.
//
// * cp.async (sm_80+): each thread copies its own element, so gathers through
//   a permutation are allowed; the copies of one commit group land together
//   and are waited for with cp_async_wait_all() followed by a CTA barrier.
// * cp.async.bulk (sm_90+): one thread copies a contiguous range (16-byte
//   aligned addresses, size a multiple of 16) through the tensor memory
//   accelerator; completion is counted in bytes on a shared-memory mbarrier.
//   Every wait on an mbarrier is bounded: after kMbarSpinLimit polls it gives
//   up and reports failure instead of spinning forever.
#pragma once
#include <cstdint>

namespace gmpm {

template <int N>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    static_assert(N == 4 || N == 8 || N == 16, "cp.async copies 4, 8 or 16 bytes");
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(N) : "memory");
}

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
    cp_async<sizeof(T)>(smem, gmem);
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ---- mbarrier + bulk copies ------------------------------------------------

constexpr int kMbarSpinLimit = 1 << 22;  // polls (each with a short sleep) before a wait gives up

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(a), "r"(count) : "memory");
}

// Make mbarrier initialisation visible to the asynchronous proxy.
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(a), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    unsigned ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (int i = 0; i < kMbarSpinLimit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        __nanosleep(64);
    }
    return false;
}

// Order this thread's earlier generic-proxy shared-memory accesses before
// later asynchronous-proxy (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// Bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) from
// global to this CTA's shared memory, completing on bar.
__device__ __forceinline__ void bulk_copy_g2s(void* smem, const void* gmem, unsigned bytes, uint64_t* bar) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(s),
        "l"(gmem), "r"(bytes), "r"(b)
        : "memory");
}

}  // namespace gmpm
