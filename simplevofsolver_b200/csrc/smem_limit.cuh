// Dynamic shared-memory limits of the kernels whose tiles depend on the grid.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

// Raises func's dynamic shared-memory limit to at least `bytes` on the current
// device.  The limit is an attribute of the function, shared by every solver
// of the process on that device, so it only ever grows: a solver set up later
// with shorter lines must not take away what an earlier one launches with.
// Called for every size, small ones included, since the default limit also
// counts the kernel's static shared memory.
inline cudaError_t raise_smem_limit(const void *func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> granted;  // (device, function)
  int dev = 0;
  const cudaError_t de = cudaGetDevice(&dev);
  if (cudaSuccess != de) return de;
  std::lock_guard<std::mutex> lock(mu);
  size_t &g = granted[{dev, func}];
  if (bytes <= g) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (cudaSuccess == e) g = bytes;
  return e;
}

template <class... A>
inline cudaError_t raise_smem_limit(void (*func)(A...), size_t bytes) {
  return raise_smem_limit(reinterpret_cast<const void *>(func), bytes);
}
