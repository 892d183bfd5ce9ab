// Host helpers shared by the kernel launchers.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace p2 {

// Raises a kernel's dynamic shared-memory limit on the current device once
// (the attribute persists for the context), so that later launches -- and
// launches recorded into a CUDA graph -- make no attribute calls.
inline cudaError_t ensure_smem(const void* func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  int& cur = done[{func, dev}];
  if (cur >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

}  // namespace p2
