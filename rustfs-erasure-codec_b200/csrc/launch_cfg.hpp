// launch_cfg.hpp -- kernel launch settings resolved once per process.
//
// A kernel's dynamic shared-memory limit is raised only when a launch needs
// more than was set before, and its occupancy is queried once per (device,
// kernel, threads, shared memory): both would otherwise run at every call,
// host time on the path of every launch.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

namespace rsgpu {

// SMs of the current device (queried once per device).
inline int device_sm_count() {
  static std::mutex mu;
  static std::map<int, int> sms;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  std::lock_guard<std::mutex> g(mu);
  auto it = sms.find(dev);
  if (it != sms.end()) return it->second;
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 1;
  sms[dev] = n;
  return n;
}

// Makes `fn` launchable with `smem` bytes of dynamic shared memory.
inline cudaError_t ensure_smem_limit(const void *fn, size_t smem) {
  if (smem <= 48 * 1024) return cudaSuccess;
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, size_t> limit;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  size_t &cur = limit[{dev, fn}];
  if (smem <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e == cudaSuccess) cur = smem;
  return e;
}

// Resident CTAs per SM of `fn` at this block size and shared memory (after
// ensure_smem_limit).
inline cudaError_t blocks_per_sm(const void *fn, int threads, size_t smem, int *out) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void *, int, size_t>, int> occ;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_tuple(dev, fn, threads, smem);
  auto it = occ.find(key);
  if (it != occ.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, fn, threads, smem);
  if (e == cudaSuccess) occ[key] = *out;
  return e;
}

}  // namespace rsgpu
