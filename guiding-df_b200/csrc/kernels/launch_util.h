// launch_util.h -- host helpers shared by the kernel launchers.
#pragma once

#include <mutex>

#include <cuda_runtime.h>

namespace gdf {

// Lets `kern` launch with as much dynamic shared memory as the device allows
// it (the per-block opt-in limit less the kernel's static shared memory).
// The attribute is process-wide per function, so it is raised once to that
// fixed ceiling rather than set to the size of the launch at hand: a graph
// kernel node of a larger size stays updatable after a smaller launch was
// set up, and launchers on other host threads never lower it under each
// other.
inline cudaError_t allow_dynamic_smem_fn(const void* kern) {
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, kern);
  if (e != cudaSuccess) return e;
  int dev = 0, optin = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
  const int ceiling = optin - static_cast<int>(a.sharedSizeBytes);
  if (a.maxDynamicSharedSizeBytes >= ceiling) return cudaSuccess;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, ceiling);
}

template <class K>
inline cudaError_t allow_dynamic_smem(K* kern) {
  return allow_dynamic_smem_fn(reinterpret_cast<const void*>(kern));
}

}  // namespace gdf
