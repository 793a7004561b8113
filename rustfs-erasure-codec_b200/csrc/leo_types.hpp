// leo_types.hpp -- launch descriptors of the Leopard tile kernels, shared by
// the host runtime (leopard.cu, batch.cu) and the device code (leo_tile.cuh).
#pragma once

#include <cstdint>

namespace rsgpu {

constexpr int kRowWords = 16;  // one 64-byte block per lane row

// One stripe of a Leopard launch.
struct LeoJob {
  uint32_t ptr_off;     // into the pointer table: k + p shard pointers
  uint32_t flag_idx;    // verify flag
  const uint16_t *err;  // decode: error locators (n entries)
  const uint8_t *role;  // decode: per shard 0 absent, 1 present (input), 2 target (output)
  uint32_t input_count;
  uint32_t pad;
};

// Geometry and tables of one Leopard codec's launch.
struct LeoArgs {
  const LeoJob *jobs;
  const uint8_t *const *ptrs;
  const uint16_t *skew;
  const uint32_t *bank;
  uint32_t *flags;
  uint32_t *scratch;  // global work rows when the lanes do not fit on chip
  uint64_t len;       // bytes per shard (multiple of 64)
  uint32_t n_jobs;
  uint32_t k, p, m, n;  // n: decode lanes (pow2 >= m + k)
  uint32_t mtrunc, last;
  uint32_t nb;     // 64-byte column blocks per tile
  uint32_t lanes;  // rows per tile (encode 2m, decode n)
  uint32_t mod;
  // Register-stage transforms (leo_fft.cuh): their multiplier tables and the
  // stage plans of the encoder IFFT / FFT over m lanes and the decoder IFFT /
  // FFT over n lanes.  Stage s of a plan is byte s of its word (log2
  // lanes-per-thread | log2 dm << 3); packed words, not byte arrays, so that
  // device code indexes them with shifts instead of a local-memory copy.
  const uint32_t *kbank;
  const uint32_t *sktab;  // kbank's tables of each skew entry (entry i: log skew[i])
  uint32_t st_ienc, st_fenc, st_idec, st_fdec;
  uint32_t n_ienc, n_fenc, n_idec, n_fdec;
};

}  // namespace rsgpu
