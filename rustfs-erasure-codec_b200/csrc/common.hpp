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
// tables" (see pack_tables()).  A verify job with verify_store set also
// writes the recomputed outputs to the n_out pointers that follow the stored
// parity (verify_with_buffer).
struct JobDesc {
  uint32_t ptr_off;
  uint16_t n_in;
  uint16_t n_out;
  uint32_t flag_idx;    // verify: index of this stripe's mismatch flag
  uint32_t verify_store;
  uint64_t vec_len;     // prefix handled by the 128-bit path (0 when misaligned)
  const uint32_t *tbl;  // packed nibble tables of this stripe's coefficient rows
};
static_assert(sizeof(JobDesc) == 32, "JobDesc layout");

// Packed table layout for one coefficient matrix of n_out x n_in: for each
// group g of 4 outputs and each input j, kTableWords words (byte r of a word
// belongs to output 4g+r):
//   [0, 16)   c * n          n = 0..15   (4+4 split: low nibble)
//   [16, 32)  c * (n << 4)   n = 0..15   (4+4 split: high nibble)
//   [32, 64)  c * i          i = 0..31   (5+3 split: low five bits)
//   [64, 72)  for output r: words 64+2r, 65+2r hold the bytes c_r * (h << 5),
//             h = 0..7        (5+3 split: high three bits, one byte per h)
constexpr int kTableWords = 72;
inline size_t packed_table_words(size_t n_out, size_t n_in) {
  return ((n_out + 3) / 4) * n_in * kTableWords;
}

uint64_t launch_counter_add(uint64_t n);

// Stream-ordered device memory from the library's own pool on the current
// device, which keeps up to 2 GiB of freed memory mapped between calls (the
// device's default pool gives freed memory back at every synchronization,
// so each call would map it afresh: host time that varied fivefold between
// passes of the same per-stripe calls).  Released with cudaFreeAsync.
// Returns a cudaError_t value.
int lib_malloc_async(void **p, size_t bytes, void *stream);
template <class T>
inline int lib_malloc_async(T **p, size_t bytes, void *stream) {
  return lib_malloc_async(reinterpret_cast<void **>(p), bytes, stream);
}
// The pool itself (cudaMemPool_t), for cudaMallocFromPoolAsync callers.
int lib_pool(void **out);
// Host -> device copy, stream-ordered on `stream`, through a pinned bounce
// buffer of the calling thread (never blocks on the stream's earlier work).
// Returns an RSGPU_* code.
int upload_to(void *dst, const void *src, size_t bytes, void *stream);
// At least n free bounce buffers of `bytes` in the calling thread's pool.
int upload_prewarm(size_t n, size_t bytes);

}  // namespace rsgpu
