// Host-side launch helpers shared by the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace pbs {

// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device; the driver call is made once per kernel, device and size.
inline cudaError_t set_smem_limit(const void* func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = done[{func, dev}];
    if (have >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e == cudaSuccess) have = bytes;
    return e;
}

}  // namespace pbs
