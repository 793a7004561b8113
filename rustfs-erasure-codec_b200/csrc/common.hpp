// common.hpp -- types shared by the host runtime and the sm_100a kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include "rsgpu.h"

namespace rsgpu {

// Bytes of columns one CTA of the classic matrix-apply kernel covers per tile:
// 256 threads x 16 bytes (one 128-bit vector per input shard per thread).
constexpr int kApplyThreads = 256;
constexpr int kApplyVec = 16;
constexpr uint64_t kApplyTile = uint64_t(kApplyThreads) * kApplyVec;

// One stripe's matrix application: out[r] = sum_j c[r][j] * in[j] over GF(2^8).
// Pointers live in a shared pointer table: ptrs[ptr_off .. ptr_off+n_in) are
// the inputs and the next n_out entries the outputs (or, for verify, the
// stored parity to compare against).  Coefficients are pre-packed "nibble
// tables" (see pack_tables()).
struct JobDesc {
  uint32_t ptr_off;
  uint16_t n_in;
  uint16_t n_out;
  uint32_t flag_idx;    // verify: index of this stripe's mismatch flag
  uint32_t reserved;
  uint64_t vec_len;     // prefix handled by the 128-bit path (0 when misaligned)
  const uint32_t *tbl;  // packed nibble tables of this stripe's coefficient rows
};
static_assert(sizeof(JobDesc) == 32, "JobDesc layout");

// Packed table layout for one coefficient matrix of n_out x n_in:
// for each group g of 4 outputs, for each input j, 32 words:
//   word n      (n < 16): bytes r = c[4g+r][j] * n          (low nibble)
//   word 16 + n (n < 16): bytes r = c[4g+r][j] * (n << 4)   (high nibble)
inline size_t packed_table_words(size_t n_out, size_t n_in) {
  return ((n_out + 3) / 4) * n_in * 32;
}

uint64_t launch_counter_add(uint64_t n);

}  // namespace rsgpu
