// launch_util.h -- the dynamic shared-memory limit of a kernel, raised only.
//
// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) holds per kernel and device for the
// whole process, and every trainer, batch and server sets it for its own K.  Setting it
// to a smaller value would break the launches of an object with a larger K that already
// exists, so the limit is only ever raised.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace lda {

inline cudaError_t raise_smem_limit(const void* fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limits;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = limits[{dev, fn}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

}  // namespace lda
