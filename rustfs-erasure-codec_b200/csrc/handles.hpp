// handles.hpp -- the opaque C handles of include/rsgpu.h that more than one
// translation unit needs to see inside.
#pragma once

#include <cuda_runtime.h>

#include <mutex>

#include "codec.hpp"
#include "rsgpu.h"

struct rsgpu_codec {
  rsgpu::Codec c;
  // internal streams for host-memory staging
  cudaStream_t io[2] = {nullptr, nullptr};
  std::mutex io_mu;
};
