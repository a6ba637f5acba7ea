// Kernel launch with its own status.
//
// A <<<>>> launch reports through cudaGetLastError, which also returns (and
// clears) an error left pending by an earlier, unrelated launch of the
// caller.  cudaLaunchKernel returns the status of this launch alone.
#pragma once
#include <cuda_runtime.h>

#include <tuple>
#include <type_traits>
#include <utility>

namespace gmpm {

template <typename... P, typename... A>
inline cudaError_t launch_kernel(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                 A&&... args) {
    static_assert(sizeof...(P) == sizeof...(A), "launch_kernel: argument count differs from the kernel's");
    std::tuple<std::decay_t<P>...> params(std::forward<A>(args)...);
    return std::apply(
        [&](auto&... p) {
            void* ptrs[] = {static_cast<void*>(&p)...};
            return cudaLaunchKernel(reinterpret_cast<const void*>(kernel), grid, block, ptrs, smem, stream);
        },
        params);
}

}  // namespace gmpm
