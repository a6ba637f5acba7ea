// Asynchronous global -> shared copies (cp.async, sm_80+ PTX).  Each thread
// copies its own element, so gathers through a permutation are allowed; the
// copies of one commit group land together and are waited for with
// cp_async_wait_all() followed by a CTA barrier.
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

}  // namespace gmpm
