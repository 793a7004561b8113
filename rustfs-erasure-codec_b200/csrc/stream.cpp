// stream.cpp -- block streaming calls (src/core/stream.rs:650-1000) over
// caller-supplied read / write callbacks.
//
// Semantics follow the reference: the block size is clamped to [1 KiB,
// 16 MiB]; each stream is read until the block is full or the stream ends;
// encode zero-pads shorter data streams to the longest one of the block;
// verify and reconstruct require every read stream of a block to return the
// same length (else IncorrectShardSize with the first offending index);
// counts, codec family and (for reconstruct) reader/writer layout are checked
// before any I/O; Leopard codecs get UnsupportedCodecFamily (the reference's
// streaming path is classic-only, and it exists for galois_8 only, so the
// tower field codec is rejected the same way).
//
// GPU pipeline: two pinned host blocks and two device blocks.  While the GPU
// encodes / verifies / rebuilds block i (upload, K1, download, event on a
// private stream), the calling thread reads block i + 1 from the callbacks,
// then writes block i's outputs once its event has fired.  Every output block
// is written before an error of a later block is returned, so the writers see
// the same prefix the reference would have written.  (Verify may read one block
// past the first mismatching block before it stops.)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "codec.hpp"
#include "handles.hpp"
#include "rsgpu.h"

namespace rsgpu {
namespace {

constexpr size_t kMinBlock = 1024, kMaxBlock = 16u << 20;

#define ST_CUDA(expr)                              \
  do {                                             \
    cudaError_t e_ = (expr);                       \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

struct Status {
  rsgpu_stream_status *out;
  int32_t codec(int32_t code, size_t shard) {
    if (out) *out = rsgpu_stream_status{RSGPU_STREAM_CODEC, code, shard};
    return code;
  }
  int32_t io(int kind, int64_t code, size_t shard) {
    if (out) *out = rsgpu_stream_status{kind, int32_t(code), shard};
    return RSGPU_ERR_STREAM_IO;
  }
  int32_t ok() {
    if (out) *out = rsgpu_stream_status{RSGPU_STREAM_OK, 0, 0};
    return RSGPU_OK;
  }
};

// Read until `cap` bytes or the end of the stream; returns the count or the
// callback's negative error.
int64_t read_full(rsgpu_read_fn rd, void *ctx, size_t shard, uint8_t *buf, size_t cap) {
  size_t total = 0;
  while (total < cap) {
    const int64_t r = rd(ctx, shard, buf + total, cap - total);
    if (r < 0) return r;
    if (r == 0) break;
    total += size_t(r);
  }
  return int64_t(total);
}

int32_t count_check(size_t actual, size_t expected, Status &st) {
  if (actual < expected) return st.codec(RSGPU_ERR_TOO_FEW_SHARDS, 0);
  if (actual > expected) return st.codec(RSGPU_ERR_TOO_MANY_SHARDS, 0);
  return RSGPU_OK;
}

bool streamable(const Codec &c) { return c.family == RSGPU_FAMILY_CLASSIC && c.field == RSGPU_FIELD_GF8; }

// Double-buffered staging of `rows` rows of `block` bytes.
struct Stage {
  size_t rows = 0, block = 0;
  uint8_t *h[2] = {nullptr, nullptr};
  uint8_t *d[2] = {nullptr, nullptr};
  uint32_t *flag_d[2] = {nullptr, nullptr};
  uint32_t *flag_h = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaStream_t s = nullptr;
  ~Stage() {
    if (s) cudaStreamSynchronize(s);
    for (int i = 0; i < 2; ++i) {
      if (h[i]) cudaFreeHost(h[i]);
      if (d[i]) cudaFree(d[i]);
      if (flag_d[i]) cudaFree(flag_d[i]);
      if (ev[i]) cudaEventDestroy(ev[i]);
    }
    if (flag_h) cudaFreeHost(flag_h);
    if (s) cudaStreamDestroy(s);
  }
  int init(size_t r, size_t b) {
    rows = r;
    block = b;
    ST_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      ST_CUDA(cudaMallocHost(&h[i], rows * block));
      ST_CUDA(cudaMalloc(&d[i], rows * block));
      ST_CUDA(cudaMalloc(&flag_d[i], 4));
      ST_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    }
    ST_CUDA(cudaMallocHost(&flag_h, 8));
    return RSGPU_OK;
  }
  uint8_t *hrow(int slot, size_t r) { return h[slot] + r * block; }
  uint8_t *drow(int slot, size_t r) { return d[slot] + r * block; }
};

}  // namespace

// ------------------------------------------------------------------ encode
int32_t encode_stream(Codec &c, size_t n_data, rsgpu_read_fn rd, void *rctx, size_t n_parity, rsgpu_write_fn wr,
                      void *wctx, size_t block_opt, rsgpu_stream_status *status) {
  Status st{status};
  if (!streamable(c)) return st.codec(RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY, 0);
  int32_t rc = count_check(n_data, c.k, st);
  if (rc) return rc;
  if ((rc = count_check(n_parity, c.m, st))) return rc;
  const size_t block = std::min(std::max(block_opt, kMinBlock), kMaxBlock);
  const size_t k = c.k, m = c.m, total = k + m;
  Stage S;
  if ((rc = S.init(total, block))) return st.codec(rc, 0);
  int pending = -1;
  size_t pending_len = 0;
  // Write block `slot`'s parity once its device work has finished.
  auto flush = [&](int slot, size_t len) -> int32_t {
    cudaError_t e = cudaEventSynchronize(S.ev[slot]);
    if (e != cudaSuccess) return st.codec(cuda_status(e), 0);
    for (size_t r = 0; r < m; ++r) {
      const int64_t w = wr(wctx, k + r, S.hrow(slot, k + r), len);
      if (w < 0) return st.io(RSGPU_STREAM_WRITE, w, k + r);
    }
    return RSGPU_OK;
  };
  for (uint64_t blk = 0;; ++blk) {
    const int slot = int(blk & 1);
    size_t actual = 0;
    std::vector<size_t> lens(k);
    for (size_t j = 0; j < k; ++j) {
      const int64_t r = read_full(rd, rctx, j, S.hrow(slot, j), block);
      if (r < 0) {
        if (pending >= 0 && (rc = flush(pending, pending_len))) return rc;
        return st.io(RSGPU_STREAM_READ, r, j);
      }
      lens[j] = size_t(r);
      actual = std::max(actual, lens[j]);
    }
    if (actual == 0) break;
    for (size_t j = 0; j < k; ++j)
      if (lens[j] < actual) std::memset(S.hrow(slot, j) + lens[j], 0, actual - lens[j]);
    std::vector<uint8_t *> ptrs(total);
    for (size_t j = 0; j < total; ++j) ptrs[j] = S.drow(slot, j);
    for (size_t j = 0; j < k; ++j)
      ST_CUDA(cudaMemcpyAsync(ptrs[j], S.hrow(slot, j), actual, cudaMemcpyHostToDevice, S.s));
    if ((rc = c.encode_dev(1, ptrs.data(), actual, S.s))) return st.codec(rc, 0);
    for (size_t r = 0; r < m; ++r)
      ST_CUDA(cudaMemcpyAsync(S.hrow(slot, k + r), ptrs[k + r], actual, cudaMemcpyDeviceToHost, S.s));
    ST_CUDA(cudaEventRecord(S.ev[slot], S.s));
    if (pending >= 0 && (rc = flush(pending, pending_len))) return rc;
    pending = slot;
    pending_len = actual;
  }
  if (pending >= 0 && (rc = flush(pending, pending_len))) return rc;
  return st.ok();
}

// ------------------------------------------------------------------ verify
int32_t verify_stream(Codec &c, size_t n_shards, rsgpu_read_fn rd, void *rctx, size_t block_opt, int32_t *ok,
                      rsgpu_stream_status *status) {
  Status st{status};
  if (!streamable(c)) return st.codec(RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY, 0);
  const size_t k = c.k, total = c.k + c.m;
  int32_t rc = count_check(n_shards, total, st);
  if (rc) return rc;
  const size_t block = std::min(std::max(block_opt, kMinBlock), kMaxBlock);
  Stage S;
  if ((rc = S.init(total, block))) return st.codec(rc, 0);
  *ok = 1;
  int pending = -1;
  // Result of block `slot`: true when its parity matched.
  auto result = [&](int slot, bool *match) -> int32_t {
    cudaError_t e = cudaEventSynchronize(S.ev[slot]);
    if (e != cudaSuccess) return st.codec(cuda_status(e), 0);
    *match = S.flag_h[slot] == 0;
    return RSGPU_OK;
  };
  for (uint64_t blk = 0;; ++blk) {
    const int slot = int(blk & 1);
    std::vector<size_t> lens(total);
    size_t actual = 0;
    int64_t read_err = 0;
    size_t err_shard = 0;
    for (size_t j = 0; j < total && !read_err; ++j) {
      const int64_t r = read_full(rd, rctx, j, S.hrow(slot, j), block);
      if (r < 0) {
        read_err = r;
        err_shard = j;
        break;
      }
      lens[j] = size_t(r);
      actual = std::max(actual, lens[j]);
    }
    // The previous block's verdict comes first: the reference stops there.
    if (pending >= 0) {
      bool match = true;
      if ((rc = result(pending, &match))) return rc;
      pending = -1;
      if (!match) {
        *ok = 0;
        return st.ok();
      }
    }
    if (read_err) return st.io(RSGPU_STREAM_READ, read_err, err_shard);
    if (actual == 0) break;
    for (size_t j = 0; j < total; ++j)
      if (lens[j] != actual) return st.codec(RSGPU_ERR_INCORRECT_SHARD_SIZE, j);
    std::vector<uint8_t *> ptrs(total);
    for (size_t j = 0; j < total; ++j) {
      ptrs[j] = S.drow(slot, j);
      ST_CUDA(cudaMemcpyAsync(ptrs[j], S.hrow(slot, j), actual, cudaMemcpyHostToDevice, S.s));
    }
    ST_CUDA(cudaMemsetAsync(S.flag_d[slot], 0, 4, S.s));
    if ((rc = c.verify_dev_async(1, ptrs.data(), actual, S.flag_d[slot], S.s))) return st.codec(rc, 0);
    ST_CUDA(cudaMemcpyAsync(S.flag_h + slot, S.flag_d[slot], 4, cudaMemcpyDeviceToHost, S.s));
    ST_CUDA(cudaEventRecord(S.ev[slot], S.s));
    pending = slot;
    (void)k;
  }
  return st.ok();
}

// ------------------------------------------------------------------ reconstruct
int32_t reconstruct_stream_from(Codec &c, size_t n_shards, const uint8_t *has_reader, rsgpu_read_fn rd, void *rctx,
                                const uint8_t *has_writer, rsgpu_write_fn wr, void *wctx, size_t block_opt,
                                rsgpu_stream_status *status) {
  Status st{status};
  const size_t total = c.k + c.m;
  int32_t rc = count_check(n_shards, total, st);
  if (rc) return rc;
  if (!streamable(c)) return st.codec(RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY, 0);
  std::vector<uint8_t> present(total);
  std::vector<size_t> missing;
  for (size_t i = 0; i < total; ++i) {
    if ((has_reader[i] != 0) == (has_writer[i] != 0)) return st.codec(RSGPU_ERR_INVALID_SHARD_FLAGS, i);
    present[i] = has_reader[i] ? 1 : 0;
    if (!present[i]) missing.push_back(i);
  }
  if (total - missing.size() < c.k) return st.codec(RSGPU_ERR_TOO_FEW_SHARDS_PRESENT, 0);
  const size_t block = std::min(std::max(block_opt, kMinBlock), kMaxBlock);
  Stage S;
  if ((rc = S.init(total, block))) return st.codec(rc, 0);
  int pending = -1;
  size_t pending_len = 0;
  auto flush = [&](int slot, size_t len) -> int32_t {
    cudaError_t e = cudaEventSynchronize(S.ev[slot]);
    if (e != cudaSuccess) return st.codec(cuda_status(e), 0);
    for (size_t i : missing) {
      const int64_t w = wr(wctx, i, S.hrow(slot, i), len);
      if (w < 0) return st.io(RSGPU_STREAM_WRITE, w, i);
    }
    return RSGPU_OK;
  };
  for (uint64_t blk = 0;; ++blk) {
    const int slot = int(blk & 1);
    size_t actual = 0;
    std::vector<size_t> lens(total, 0);
    for (size_t i = 0; i < total; ++i) {
      if (!present[i]) continue;
      const int64_t r = read_full(rd, rctx, i, S.hrow(slot, i), block);
      if (r < 0) {
        if (pending >= 0 && (rc = flush(pending, pending_len))) return rc;
        return st.io(RSGPU_STREAM_READ, r, i);
      }
      lens[i] = size_t(r);
      actual = std::max(actual, lens[i]);
    }
    if (pending >= 0) {
      if ((rc = flush(pending, pending_len))) return rc;
      pending = -1;
    }
    if (actual == 0) break;
    for (size_t i = 0; i < total; ++i)
      if (present[i] && lens[i] != actual) return st.codec(RSGPU_ERR_INCORRECT_SHARD_SIZE, i);
    std::vector<uint8_t *> ptrs(total);
    for (size_t i = 0; i < total; ++i) {
      ptrs[i] = S.drow(slot, i);
      if (present[i]) ST_CUDA(cudaMemcpyAsync(ptrs[i], S.hrow(slot, i), actual, cudaMemcpyHostToDevice, S.s));
    }
    rc = c.reconstruct_dev(1, ptrs.data(), present.data(), actual, RSGPU_GOAL_ALL, nullptr, 0, S.s);
    if (rc) return st.codec(rc, 0);
    for (size_t i : missing)
      ST_CUDA(cudaMemcpyAsync(S.hrow(slot, i), ptrs[i], actual, cudaMemcpyDeviceToHost, S.s));
    ST_CUDA(cudaEventRecord(S.ev[slot], S.s));
    pending = slot;
    pending_len = actual;
  }
  return st.ok();
}

}  // namespace rsgpu

extern "C" {

void rsgpu_stream_options_default(rsgpu_stream_options *out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->block_size = 4u << 20;
}

static size_t block_of(const rsgpu_stream_options *o) { return o ? o->block_size : (4u << 20); }

int32_t rsgpu_encode_stream(const rsgpu_codec *codec, size_t n_data, rsgpu_read_fn read, void *read_ctx,
                            size_t n_parity, rsgpu_write_fn write, void *write_ctx, const rsgpu_stream_options *opts,
                            rsgpu_stream_status *status) {
  if (!codec || !read || !write) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::encode_stream(const_cast<rsgpu_codec *>(codec)->c, n_data, read, read_ctx, n_parity, write,
                              write_ctx, block_of(opts), status);
}

int32_t rsgpu_verify_stream(const rsgpu_codec *codec, size_t n_shards, rsgpu_read_fn read, void *read_ctx,
                            const rsgpu_stream_options *opts, int32_t *ok, rsgpu_stream_status *status) {
  if (!codec || !read || !ok) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::verify_stream(const_cast<rsgpu_codec *>(codec)->c, n_shards, read, read_ctx, block_of(opts), ok,
                              status);
}

int32_t rsgpu_reconstruct_stream_from(const rsgpu_codec *codec, size_t n_shards, const uint8_t *has_reader,
                                      rsgpu_read_fn read, void *read_ctx, const uint8_t *has_writer,
                                      rsgpu_write_fn write, void *write_ctx, const rsgpu_stream_options *opts,
                                      rsgpu_stream_status *status) {
  if (!codec || !has_reader || !has_writer || !read || !write) return RSGPU_ERR_INVALID_ARGUMENT;
  return rsgpu::reconstruct_stream_from(const_cast<rsgpu_codec *>(codec)->c, n_shards, has_reader, read, read_ctx,
                                        has_writer, write, write_ctx, block_of(opts), status);
}

}  // extern "C"
