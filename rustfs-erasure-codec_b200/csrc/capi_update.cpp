// capi_update.cpp -- incremental parity (encode_single, encode_single_sep,
// update), split / join and the encoding-format stable identity.
//
// encode_single / update run on the matrix-apply kernels with accumulating
// outputs (K1 for GF(2^8), the tower kernel for galois_16): parity_r (+)=
// sum_j c[k + r][j] * in_j, one read of each input and one read-modify-write
// of each parity shard.  split / join and the format identity are host-side
// byte layout helpers with no device work.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "codec.hpp"
#include "handles.hpp"
#include "leopard.hpp"
#include "rsgpu.h"

using rsgpu::Codec;

namespace {

#define UP_CUDA(expr)                                      \
  do {                                                     \
    cudaError_t e_ = (expr);                               \
    if (e_ != cudaSuccess) return rsgpu::cuda_status(e_);  \
  } while (0)

bool is_leopard(const Codec &c) { return c.family != RSGPU_FAMILY_CLASSIC; }
bool is_tower(const Codec &c) { return c.family == RSGPU_FAMILY_CLASSIC && c.field != RSGPU_FIELD_GF8; }
size_t elem_width(const Codec &c) { return is_tower(c) ? 2 : 1; }

// check_slices!(multi => lens): src/macros.rs:142-155.
int check_multi(const size_t *lens, size_t n) {
  if (n == 0) return RSGPU_OK;
  if (lens[0] == 0) return RSGPU_ERR_EMPTY_SHARD;
  for (size_t i = 0; i < n; ++i)
    if (lens[i] != lens[0]) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  return RSGPU_OK;
}

int check_count(size_t n, size_t want, int too_few, int too_many) {
  if (n < want) return too_few;
  if (n > want) return too_many;
  return RSGPU_OK;
}

// parity (+)= sum_j c[k + r][cols[j]] * inputs[j] on device pointers.
int apply(Codec &c, const std::vector<const uint8_t *> &in, const std::vector<size_t> &cols, uint8_t *const *parity,
          size_t len, bool accumulate, cudaStream_t s) {
  if (is_tower(c)) return rsgpu::tower_apply_columns(c, in, cols, parity, len, accumulate, s);
  return c.apply_parity_columns(in, cols, parity, len, accumulate, s);
}

// Host-memory form: stage inputs and parity through the device, compute,
// copy the parity back and wait.
int apply_host(Codec &c, const std::vector<const uint8_t *> &in, const std::vector<size_t> &cols,
               uint8_t *const *parity, size_t len, bool accumulate) {
  const size_t n_in = in.size(), m = c.m;
  cudaStream_t s = nullptr;
  UP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  uint8_t *d = nullptr;
  const size_t pitch = (len + 255) & ~size_t(255);
  cudaError_t e = cudaError_t(rsgpu::lib_malloc_async(reinterpret_cast<void **>(&d), (n_in + m) * pitch, s));
  int rc = e == cudaSuccess ? RSGPU_OK : rsgpu::cuda_status(e);
  std::vector<const uint8_t *> din(n_in);
  std::vector<uint8_t *> dpar(m);
  for (size_t j = 0; j < n_in && rc == RSGPU_OK; ++j) {
    din[j] = d + j * pitch;
    if (cudaMemcpyAsync(const_cast<uint8_t *>(din[j]), in[j], len, cudaMemcpyHostToDevice, s) != cudaSuccess)
      rc = RSGPU_ERR_CUDA;
  }
  for (size_t r = 0; r < m && rc == RSGPU_OK; ++r) {
    dpar[r] = d + (n_in + r) * pitch;
    if (accumulate &&
        cudaMemcpyAsync(dpar[r], parity[r], len, cudaMemcpyHostToDevice, s) != cudaSuccess)
      rc = RSGPU_ERR_CUDA;
  }
  if (rc == RSGPU_OK) rc = apply(c, din, cols, dpar.data(), len, accumulate, s);
  for (size_t r = 0; r < m && rc == RSGPU_OK; ++r)
    if (cudaMemcpyAsync(parity[r], dpar[r], len, cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = RSGPU_ERR_CUDA;
  if (d) cudaFreeAsync(d, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && rc == RSGPU_OK) rc = RSGPU_ERR_CUDA;
  cudaStreamDestroy(s);
  return rc;
}

int run(Codec &c, const std::vector<const uint8_t *> &in, const std::vector<size_t> &cols, uint8_t *const *parity,
        size_t len, bool accumulate, int32_t mem, void *stream) {
  if (mem == RSGPU_MEM_DEVICE)
    return apply(c, in, cols, parity, len, accumulate, static_cast<cudaStream_t>(stream));
  if (mem != RSGPU_MEM_HOST) return RSGPU_ERR_INVALID_ARGUMENT;
  return apply_host(c, in, cols, parity, len, accumulate);
}

int single(Codec &c, size_t i_data, const uint8_t *data, uint8_t *const *parity, size_t len, int32_t mem,
           void *stream) {
  if (len % elem_width(c)) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  // src/core/encode.rs code_single_slice: shard 0 overwrites, later shards add.
  return run(c, {data}, {i_data}, parity, len, i_data != 0, mem, stream);
}

}  // namespace

extern "C" {

int32_t rsgpu_encode_single(const rsgpu_codec *hc, size_t i_data, uint8_t *const *shards, const size_t *lens,
                            size_t n, int32_t mem, void *stream) {
  if (!hc || (!shards && n) || (!lens && n)) return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = const_cast<rsgpu_codec *>(hc)->c;
  // src/core/encode.rs:892-908: family, index, piece count, slices.
  if (is_leopard(c)) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  if (i_data >= c.k) return RSGPU_ERR_INVALID_INDEX;
  int rc = check_count(n, c.k + c.m, RSGPU_ERR_TOO_FEW_SHARDS, RSGPU_ERR_TOO_MANY_SHARDS);
  if (rc || (rc = check_multi(lens, n))) return rc;
  return single(c, i_data, shards[i_data], shards + c.k, lens[0], mem, stream);
}

int32_t rsgpu_encode_single_sep(const rsgpu_codec *hc, size_t i_data, const uint8_t *data, size_t data_len,
                                uint8_t *const *parity, const size_t *parity_lens, size_t n_parity, int32_t mem,
                                void *stream) {
  if (!hc || !data || (!parity && n_parity) || (!parity_lens && n_parity)) return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = const_cast<rsgpu_codec *>(hc)->c;
  // src/core/encode.rs:912-930.
  if (is_leopard(c)) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  if (i_data >= c.k) return RSGPU_ERR_INVALID_INDEX;
  int rc = check_count(n_parity, c.m, RSGPU_ERR_TOO_FEW_PARITY_SHARDS, RSGPU_ERR_TOO_MANY_PARITY_SHARDS);
  if (rc || (rc = check_multi(parity_lens, n_parity))) return rc;
  if (parity_lens[0] != data_len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  return single(c, i_data, data, parity, data_len, mem, stream);
}

int32_t rsgpu_update(const rsgpu_codec *hc, const uint8_t *const *old_data, const size_t *old_lens, size_t n_old,
                     const uint8_t *const *new_data, const size_t *new_lens, size_t n_new, uint8_t *const *parity,
                     const size_t *parity_lens, size_t n_parity, int32_t mem, void *stream) {
  if (!hc || (!old_data && n_old) || (!old_lens && n_old) || (!new_data && n_new) || (!new_lens && n_new) ||
      (!parity && n_parity) || (!parity_lens && n_parity))
    return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = const_cast<rsgpu_codec *>(hc)->c;
  // src/core/encode.rs:1048-1080: family, counts, slices, lengths.
  if (is_leopard(c)) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  int rc = check_count(n_old, c.k, RSGPU_ERR_TOO_FEW_DATA_SHARDS, RSGPU_ERR_TOO_MANY_DATA_SHARDS);
  if (rc) return rc;
  if ((rc = check_count(n_parity, c.m, RSGPU_ERR_TOO_FEW_PARITY_SHARDS, RSGPU_ERR_TOO_MANY_PARITY_SHARDS))) return rc;
  if ((rc = check_count(n_new, c.k, RSGPU_ERR_TOO_FEW_DATA_SHARDS, RSGPU_ERR_TOO_MANY_DATA_SHARDS))) return rc;
  if ((rc = check_multi(old_lens, n_old)) || (rc = check_multi(parity_lens, n_parity))) return rc;
  if (old_lens[0] != parity_lens[0]) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  const size_t len = old_lens[0];
  if (len == 0) return RSGPU_ERR_EMPTY_SHARD;
  std::vector<const uint8_t *> in;
  std::vector<size_t> cols;
  for (size_t j = 0; j < c.k; ++j) {
    if (!new_data[j]) continue;
    if (new_lens[j] != len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
    // c * (old + new) = c * old + c * new: both go in as inputs of column j.
    in.push_back(old_data[j]);
    cols.push_back(j);
    in.push_back(new_data[j]);
    cols.push_back(j);
  }
  if (in.empty()) return RSGPU_OK;
  if (len % elem_width(c)) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  return run(c, in, cols, parity, len, true, mem, stream);
}

size_t rsgpu_split_shard_len(const rsgpu_codec *hc, size_t data_len) {
  if (!hc) return 0;
  const Codec &c = hc->c;
  // src/core/codec.rs:486-491; Leopard: src/core/leopard.rs:75-98.
  if (is_leopard(c)) {
    const size_t per = (data_len + c.k - 1) / c.k;
    const size_t rounded = std::max<size_t>((per + 63) / 64 * 64, 64);
    return rounded;
  }
  const size_t w = elem_width(c), elems = data_len / w;
  return ((elems + c.k - 1) / c.k) * w;
}

int32_t rsgpu_split(const rsgpu_codec *hc, const uint8_t *data, size_t data_len, uint8_t *out, size_t out_len) {
  if (!hc || (!data && data_len)) return RSGPU_ERR_INVALID_ARGUMENT;
  const Codec &c = hc->c;
  if (data_len % elem_width(c)) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  const size_t sl = rsgpu_split_shard_len(hc, data_len);
  if (sl == 0) return RSGPU_OK;  // classic, empty payload: k empty shards
  if (out_len < sl * c.k || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  // Shard i holds bytes [i * sl, (i + 1) * sl) of the data, zero-padded.
  for (size_t i = 0; i < c.k; ++i) {
    const size_t start = i * sl;
    const size_t n = start < data_len ? std::min(sl, data_len - start) : 0;
    if (n) std::memcpy(out + start, data + start, n);
    if (n < sl) std::memset(out + start + n, 0, sl - n);
  }
  return RSGPU_OK;
}

int32_t rsgpu_join(const rsgpu_codec *hc, const uint8_t *const *shards, const size_t *lens, size_t n, uint8_t *out,
                   size_t out_len, size_t *written) {
  if (!hc || (!shards && n) || (!lens && n) || !written) return RSGPU_ERR_INVALID_ARGUMENT;
  const Codec &c = hc->c;
  // src/core/codec.rs:509-538: data piece count, equal non-empty slices, then
  // concatenate up to out_len bytes.
  int rc = check_count(n, c.k, RSGPU_ERR_TOO_FEW_DATA_SHARDS, RSGPU_ERR_TOO_MANY_DATA_SHARDS);
  if (rc || (rc = check_multi(lens, n))) return rc;
  const size_t target = std::min(out_len, lens[0] * n);
  if (target && !out) return RSGPU_ERR_INVALID_ARGUMENT;
  size_t done = 0;
  for (size_t i = 0; i < n && done < target; ++i) {
    const size_t take = std::min(target - done, lens[i]);
    std::memcpy(out + done, shards[i], take);
    done += take;
  }
  *written = done;
  return RSGPU_OK;
}

// src/core/format.rs:168-220 (EncodingFormat::stable_id_bytes, version 1):
// magic "RSEFMT\0\0", version u16, family u8, field-id length u32 and bytes,
// element width u32, field order / data / parity / rows / cols as u64, then
// the matrix coefficients row-major; all integers big-endian.
int32_t rsgpu_format_id(const rsgpu_codec *hc, uint8_t *out, size_t cap, size_t *len) {
  if (!hc || !len) return RSGPU_ERR_INVALID_ARGUMENT;
  const Codec &c = hc->c;
  const bool tower = is_tower(c);
  const char *field_id = tower ? "rustfs.gf16.tower-11d-x2-02x-80.ax-ac.v1" : "rustfs.gf8.poly-11d.u8.v1";
  const uint32_t width = tower ? 2 : 1;
  const uint64_t order = tower ? 65536 : 256;
  // Leopard codecs carry no matrix (src/core/codec.rs:318-326).
  const uint64_t rows = is_leopard(c) ? 0 : c.k + c.m, cols = is_leopard(c) ? 0 : c.k;
  std::vector<uint8_t> b;
  const char magic[8] = {'R', 'S', 'E', 'F', 'M', 'T', 0, 0};
  b.insert(b.end(), magic, magic + 8);
  b.push_back(0);
  b.push_back(1);  // version 1
  b.push_back(uint8_t(c.family));
  auto be32 = [&](uint32_t v) {
    for (int s = 24; s >= 0; s -= 8) b.push_back(uint8_t(v >> s));
  };
  auto be64 = [&](uint64_t v) {
    for (int s = 56; s >= 0; s -= 8) b.push_back(uint8_t(v >> s));
  };
  const size_t id_len = std::strlen(field_id);
  be32(uint32_t(id_len));
  b.insert(b.end(), field_id, field_id + id_len);
  be32(width);
  for (uint64_t v : {order, uint64_t(c.k), uint64_t(c.m), rows, cols}) be64(v);
  for (uint64_t r = 0; r < rows; ++r)
    for (uint64_t j = 0; j < cols; ++j) {
      if (tower) {
        const rsgpu::T16 e = c.tmatrix[r * c.k + j];
        b.push_back(e.x);
        b.push_back(e.c);
      } else {
        b.push_back(c.matrix[r * c.k + j]);
      }
    }
  *len = b.size();
  if (!out) return RSGPU_OK;
  if (cap < b.size()) return RSGPU_ERR_INVALID_ARGUMENT;
  std::memcpy(out, b.data(), b.size());
  return RSGPU_OK;
}

}  // extern "C"
