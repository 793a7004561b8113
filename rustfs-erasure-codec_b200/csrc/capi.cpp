// capi.cpp -- the extern "C" boundary (include/rsgpu.h).
//
// Each entry point validates its arguments with the reference's error
// precedence (src/macros.rs:142-245, src/core/recovery_plan.rs:262-387,
// src/core/reconstruct.rs:795-838) before any device work, then hands device
// pointers to the Codec.  Host-memory calls are staged through device memory
// in chunks on two internal streams so that the host->device copy of one
// chunk overlaps the kernels and device->host copy of the previous one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <new>
#include <vector>

#include "codec.hpp"
#include "handles.hpp"
#include "leopard.hpp"
#include "rsgpu.h"

using rsgpu::Codec;


struct rsgpu_batch {
  rsgpu_codec *codec = nullptr;
  int op = 0;
  size_t n_stripes = 0;
  rsgpu::ApplyLaunch apply;                // classic families
  std::shared_ptr<rsgpu::LeoLaunch> leo;   // Leopard families
  uint32_t *flags = nullptr;               // verify flags (device)
  uint32_t *owned_tables = nullptr;        // private copies of the decode tables
  ~rsgpu_batch() {
    cudaDeviceSynchronize();  // no queued launch may still read the tables
    apply.release(nullptr);
    if (flags) cudaFree(flags);
    if (owned_tables) cudaFree(owned_tables);
  }
};

struct rsgpu_verify_ws {
  size_t shard_len = 0;
};

// A prepared reconstruction plan (src/core/workspace.rs:70-112): the erasure
// layout and goal it was prepared for, the preparing codec's shape and
// encoding-format identity (reuse by another codec is checked against them,
// src/core/reconstruct.rs:702-726), and for GF(2^8) codecs the plan's
// survivors with a private device copy of its decode tables, so running it
// does no cache lookup and no inversion.
struct rsgpu_reconstruct_ws {
  size_t k = 0, m = 0;
  std::vector<uint8_t> format;
  std::vector<uint8_t> present;
  size_t shard_len = 0;
  int goal = 0;
  std::vector<uint8_t> required;
  std::vector<size_t> targets;
  std::vector<uint16_t> survivors;
  uint32_t *tbl = nullptr;
  ~rsgpu_reconstruct_ws() {
    if (tbl) cudaFree(tbl);  // waits for queued work that may still read it
  }
};

namespace rsgpu {
uint64_t launch_counter();
}

namespace {

#define RS_CUDA(expr)                                 \
  do {                                                \
    cudaError_t e_ = (expr);                          \
    if (e_ != cudaSuccess) return rsgpu::cuda_status(e_); \
  } while (0)

inline cudaStream_t S(void *p) { return static_cast<cudaStream_t>(p); }

int ensure_io(rsgpu_codec *h) {
  if (!h->io[0]) {
    RS_CUDA(cudaStreamCreateWithFlags(&h->io[0], cudaStreamNonBlocking));
    RS_CUDA(cudaStreamCreateWithFlags(&h->io[1], cudaStreamNonBlocking));
  }
  return RSGPU_OK;
}

size_t round16(size_t n) { return (n + 15) & ~size_t(15); }

// Staging memory of host-memory calls comes from the library's own pool
// (lib_pool), which keeps freed memory mapped between calls.
int staging_pool(int device, cudaMemPool_t *out) {
  (void)device;  // the pool of the current device
  void *p = nullptr;
  RS_CUDA(cudaError_t(rsgpu::lib_pool(&p)));
  *out = static_cast<cudaMemPool_t>(p);
  return RSGPU_OK;
}

// Stripes per host-staging chunk: about 256 MiB of device staging each.
size_t chunk_stripes(size_t per_stripe_bytes) {
  size_t c = (256u << 20) / std::max<size_t>(per_stripe_bytes, 1);
  return std::max<size_t>(c, 1);
}

int new_codec(size_t k, size_t m, const rsgpu_options *opts, const uint8_t *custom, int field,
              rsgpu_codec **out) {
  if (!out) return RSGPU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  rsgpu_options o;
  rsgpu_options_default(&o);
  if (opts) o = *opts;
  // src/core/codec.rs:269-349 (with_options) check order.
  if (k == 0) return RSGPU_ERR_TOO_FEW_DATA_SHARDS;
  if (m == 0) return RSGPU_ERR_TOO_FEW_PARITY_SHARDS;
  const size_t total = k + m;
  if (custom && field == RSGPU_FIELD_GF8) {
    if (total > 256) return RSGPU_ERR_TOO_MANY_SHARDS;
    if (o.codec_family != RSGPU_FAMILY_CLASSIC) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
    o.matrix_mode = RSGPU_MATRIX_CUSTOM;
  } else if (field == RSGPU_FIELD_GF8) {
    o.codec_family = rsgpu::resolve_family(o.codec_family, o.leopard_mode, total, m);
    const size_t cap = o.codec_family == RSGPU_FAMILY_LEOPARD_GF16 ? 65536 : 256;
    if (total > cap) return RSGPU_ERR_TOO_MANY_SHARDS;
    int rc = rsgpu::validate_leopard_family(o.codec_family, k, m);
    if (rc) return rc;
    if (o.codec_family == RSGPU_FAMILY_CLASSIC && o.matrix_mode == RSGPU_MATRIX_CUSTOM)
      return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
  } else {
    if (total > 65536) return RSGPU_ERR_TOO_MANY_SHARDS;
    if (o.codec_family != RSGPU_FAMILY_CLASSIC) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
    if (custom) o.matrix_mode = RSGPU_MATRIX_CUSTOM;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return RSGPU_ERR_NO_DEVICE;
  rsgpu_codec *h = new (std::nothrow) rsgpu_codec();
  if (!h) return RSGPU_ERR_OUT_OF_MEMORY;
  Codec &c = h->c;
  c.k = k;
  c.m = m;
  c.opts = o;
  c.family = o.codec_family;
  c.field = field;
  int rc;
  if (field == RSGPU_FIELD_GF16_TOWER)
    rc = c.init_tower(custom);
  else if (c.family == RSGPU_FAMILY_CLASSIC)
    rc = c.init_classic(custom);
  else
    rc = c.init_leopard();
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return RSGPU_OK;
}

// ---------------------------------------------------------------- dispatch
// Device-pointer operations for any family.
int do_encode(Codec &c, size_t n, uint8_t *const *sh, size_t len, cudaStream_t s) {
  if (c.family != RSGPU_FAMILY_CLASSIC) return rsgpu::leopard_encode(c, n, sh, len, s);
  if (c.field == RSGPU_FIELD_GF16_TOWER) return rsgpu::tower_encode(c, n, sh, len, s);
  return c.encode_dev(n, sh, len, s);
}
int do_verify(Codec &c, size_t n, const uint8_t *const *sh, size_t len, uint8_t *ok, cudaStream_t s) {
  if (c.family != RSGPU_FAMILY_CLASSIC) return rsgpu::leopard_verify(c, n, sh, len, ok, s);
  if (c.field == RSGPU_FIELD_GF16_TOWER) return rsgpu::tower_verify(c, n, sh, len, ok, s);
  return c.verify_dev(n, sh, len, ok, s);
}
int do_reconstruct(Codec &c, size_t n, uint8_t *const *sh, const uint8_t *present, size_t len, int goal,
                   const uint8_t *req, size_t nreq, cudaStream_t s) {
  if (c.family != RSGPU_FAMILY_CLASSIC) return rsgpu::leopard_reconstruct(c, n, sh, present, len, goal, req, nreq, s);
  if (c.field == RSGPU_FIELD_GF16_TOWER)
    return rsgpu::tower_reconstruct(c, n, sh, present, len, goal, req, nreq, s);
  return c.reconstruct_dev(n, sh, present, len, goal, req, nreq, s);
}

// Which shards a stripe reads (in) and writes (out) for an operation.
enum Op { OP_ENCODE, OP_VERIFY, OP_RECONSTRUCT };

// Queues shard copies in one direction on one stream, merging copies that are
// contiguous on both sides into a single cudaMemcpyAsync: a stripe's shards,
// and consecutive stripes, usually sit back to back in the caller's buffer and
// in the staging area, so a chunk moves in a few large transfers.
struct CopyRun {
  cudaMemcpyKind kind;
  cudaStream_t s;
  char *dst = nullptr;
  const char *src = nullptr;
  size_t bytes = 0;
  int add(void *d, const void *from, size_t n) {
    char *dd = static_cast<char *>(d);
    const char *ss = static_cast<const char *>(from);
    if (bytes && dd == dst + bytes && ss == src + bytes) {
      bytes += n;
      return RSGPU_OK;
    }
    const int rc = flush();
    dst = dd;
    src = ss;
    bytes = n;
    return rc;
  }
  int flush() {
    if (!bytes) return RSGPU_OK;
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s);
    bytes = 0;
    return e == cudaSuccess ? RSGPU_OK : rsgpu::cuda_status(e);
  }
};

// Host-memory execution: stage chunks of stripes through device memory.
// `in_mask`/`out_mask` (per stripe, k+m flags) say which shards to copy in
// and back.
int run_host(rsgpu_codec *h, Op op, size_t n_stripes, uint8_t *const *host, const uint8_t *present, size_t len,
             int goal, const uint8_t *req, size_t nreq, uint8_t *ok, void *user_stream) {
  Codec &c = h->c;
  const size_t total = c.k + c.m;
  std::lock_guard<std::mutex> g(h->io_mu);
  int rc = ensure_io(h);
  if (rc) return rc;
  // Order after work already queued on the caller's stream.
  cudaEvent_t ev;
  RS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  RS_CUDA(cudaEventRecord(ev, S(user_stream)));
  RS_CUDA(cudaStreamWaitEvent(h->io[0], ev, 0));
  RS_CUDA(cudaStreamWaitEvent(h->io[1], ev, 0));
  // A classic GF(2^8) verify writes the mismatch flags of the whole call into
  // one device array that is read back once at the end, so no chunk waits
  // on the host for its own result before the next chunk's copies are queued.
  // The other families report per chunk.
  uint32_t *vflags = nullptr;
  if (op == OP_VERIFY && c.family == RSGPU_FAMILY_CLASSIC && c.field == RSGPU_FIELD_GF8) {
    RS_CUDA(cudaError_t(rsgpu::lib_malloc_async(reinterpret_cast<void **>(&vflags), std::max<size_t>(n_stripes, 1) * 4, h->io[0])));
    RS_CUDA(cudaMemsetAsync(vflags, 0, std::max<size_t>(n_stripes, 1) * 4, h->io[0]));
    RS_CUDA(cudaEventRecord(ev, h->io[0]));
    RS_CUDA(cudaStreamWaitEvent(h->io[1], ev, 0));
  }
  cudaEventDestroy(ev);
  const size_t pitch = round16(len);
  const size_t per = chunk_stripes(total * pitch);
  cudaMemPool_t pool = nullptr;
  if ((rc = staging_pool(c.device, &pool))) return rc;
  std::vector<uint8_t *> dptr;
  std::vector<uint8_t> in_flags(total), out_flags(total);
  int status = RSGPU_OK;
  for (size_t base = 0, ci = 0; base < n_stripes && status == RSGPU_OK; base += per, ++ci) {
    const size_t cnt = std::min(per, n_stripes - base);
    cudaStream_t s = h->io[ci & 1];
    uint8_t *stage = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&stage), cnt * total * pitch, pool, s);
    if (e != cudaSuccess) return rsgpu::cuda_status(e);
    dptr.resize(cnt * total);
    for (size_t i = 0; i < cnt * total; ++i) dptr[i] = stage + i * pitch;
    // Inputs are queued first; the job-table upload and the kernel follow them
    // on the same stream.
    // A classic rebuild reads only the first k present shards (the plan's
    // survivors, src/core/recovery_plan.rs:329-387); Leopard reads every
    // present shard.
    CopyRun up{cudaMemcpyHostToDevice, s};
    const bool first_k = c.family == RSGPU_FAMILY_CLASSIC;
    for (size_t sidx = 0; sidx < cnt; ++sidx) {
      const size_t st = base + sidx;
      size_t used = 0;
      for (size_t i = 0; i < total; ++i) {
        bool in = op == OP_ENCODE ? i < c.k : op == OP_VERIFY ? true : present[st * total + i] != 0;
        if (op == OP_RECONSTRUCT && in) in = !first_k || used++ < c.k;
        if (in && (rc = up.add(dptr[sidx * total + i], host[st * total + i], len))) return rc;
      }
    }
    if ((rc = up.flush())) return rc;
    if (op == OP_ENCODE)
      status = do_encode(c, cnt, dptr.data(), len, s);
    else if (op == OP_VERIFY)
      status = vflags ? c.verify_dev_async(cnt, dptr.data(), len, vflags + base, s)
                      : do_verify(c, cnt, const_cast<const uint8_t *const *>(dptr.data()), len, ok + base, s);
    else
      status = do_reconstruct(c, cnt, dptr.data(), present + base * total, len, goal, req, nreq, s);
    if (status == RSGPU_OK && op != OP_VERIFY) {
      CopyRun down{cudaMemcpyDeviceToHost, s};
      for (size_t sidx = 0; sidx < cnt; ++sidx) {
        const size_t st = base + sidx;
        const uint8_t *pr = op == OP_RECONSTRUCT ? present + st * total : nullptr;
        // Which missing shards are targets follows the goal.
        for (size_t i = 0; i < total; ++i) {
          bool out;
          if (op == OP_ENCODE)
            out = i >= c.k;
          else {
            out = !pr[i] && (goal == RSGPU_GOAL_ALL || (goal == RSGPU_GOAL_DATA && i < c.k) ||
                             (goal == RSGPU_GOAL_REQUIRED && i < nreq && req[i]));
          }
          if (out && (rc = down.add(host[st * total + i], dptr[sidx * total + i], len))) return rc;
        }
      }
      if ((rc = down.flush())) return rc;
    }
    RS_CUDA(cudaFreeAsync(stage, s));
  }
  RS_CUDA(cudaStreamSynchronize(h->io[0]));
  RS_CUDA(cudaStreamSynchronize(h->io[1]));
  if (vflags) {
    if (status == RSGPU_OK) {
      std::vector<uint32_t> f(n_stripes);
      RS_CUDA(cudaMemcpyAsync(f.data(), vflags, n_stripes * 4, cudaMemcpyDeviceToHost, h->io[0]));
      RS_CUDA(cudaStreamSynchronize(h->io[0]));
      for (size_t i = 0; i < n_stripes; ++i) ok[i] = f[i] ? 0 : 1;
    }
    RS_CUDA(cudaFreeAsync(vflags, h->io[0]));
  }
  if (status == RSGPU_OK) status = c.take_device_status(h->io[0]);
  return status;
}

// Host-memory form of a single-stripe call: every non-null host buffer i gets
// a device copy of lens[i] bytes, copied in when in[i] and back when out[i];
// `fn` runs on the device pointers (null where the host pointer is null) on
// the codec's first internal stream, ordered after the caller's stream, and
// the call returns once the outputs are back in host memory.
template <class F>
int run_host_single(rsgpu_codec *h, size_t n, uint8_t *const *host, const size_t *lens, const std::vector<uint8_t> &in,
                    const std::vector<uint8_t> &out, void *user_stream, F &&fn) {
  std::lock_guard<std::mutex> g(h->io_mu);
  int rc = ensure_io(h);
  if (rc) return rc;
  cudaStream_t s = h->io[0];
  cudaEvent_t ev;
  RS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  RS_CUDA(cudaEventRecord(ev, S(user_stream)));
  RS_CUDA(cudaStreamWaitEvent(s, ev, 0));
  cudaEventDestroy(ev);
  std::vector<size_t> off(n, 0);
  size_t bytes = 0;
  for (size_t i = 0; i < n; ++i) {
    off[i] = bytes;
    if (host[i]) bytes += round16(lens[i]);
  }
  cudaMemPool_t pool = nullptr;
  if ((rc = staging_pool(h->c.device, &pool))) return rc;
  uint8_t *stage = nullptr;
  RS_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&stage), std::max<size_t>(bytes, 16), pool, s));
  std::vector<uint8_t *> d(n, nullptr);
  CopyRun up{cudaMemcpyHostToDevice, s};
  for (size_t i = 0; i < n; ++i) {
    if (!host[i]) continue;
    d[i] = stage + off[i];
    if (in[i] && lens[i] && (rc = up.add(d[i], host[i], lens[i]))) return rc;
  }
  if ((rc = up.flush())) return rc;
  int status = fn(d.data(), s);
  if (status == RSGPU_OK) {
    CopyRun down{cudaMemcpyDeviceToHost, s};
    for (size_t i = 0; i < n; ++i)
      if (host[i] && out[i] && lens[i] && (rc = down.add(host[i], d[i], lens[i]))) return rc;
    if ((rc = down.flush())) return rc;
  }
  RS_CUDA(cudaFreeAsync(stage, s));
  RS_CUDA(cudaStreamSynchronize(s));
  if (status == RSGPU_OK) status = h->c.take_device_status(s);
  return status;
}

// Per-call shard validation for reconstruct (src/core/recovery_plan.rs:262-387).
int check_reconstruct(const Codec &c, const size_t *lens, const uint8_t *present, size_t n, int goal,
                      const uint8_t *required, size_t n_required, size_t *shard_len) {
  const size_t total = c.k + c.m;
  if (goal == RSGPU_GOAL_REQUIRED && n_required != c.k && n_required != total) return RSGPU_ERR_INVALID_SHARD_FLAGS;
  if (n < total) return RSGPU_ERR_TOO_FEW_SHARDS;
  if (n > total) return RSGPU_ERR_TOO_MANY_SHARDS;
  size_t len = 0, np = 0;
  const bool leopard = c.family != RSGPU_FAMILY_CLASSIC;
  for (size_t i = 0; i < n; ++i) {
    if (!present[i]) continue;
    if (lens[i] == 0) return RSGPU_ERR_EMPTY_SHARD;
    if ((len && lens[i] != len) || (leopard && lens[i] % 64)) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
    len = lens[i];
    ++np;
  }
  if (np < c.k) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
  if (np == total) {
    *shard_len = 0;  // nothing to do
    return RSGPU_OK;
  }
  if (c.field == RSGPU_FIELD_GF16_TOWER && len % 2) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  // A missing target must come with a buffer of the shard length (ShardSlot
  // semantics, src/lib.rs:377-406).
  for (size_t i = 0; i < n; ++i) {
    if (present[i]) continue;
    bool target = goal == RSGPU_GOAL_ALL || (goal == RSGPU_GOAL_DATA && i < c.k) ||
                  (goal == RSGPU_GOAL_REQUIRED && i < n_required && required[i]);
    if (target && lens[i] < len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  }
  *shard_len = len;
  return RSGPU_OK;
}

int check_family_len(const Codec &c, size_t len) {
  if (c.family != RSGPU_FAMILY_CLASSIC && (len % 64)) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  if (c.field == RSGPU_FIELD_GF16_TOWER && (len % 2)) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  return RSGPU_OK;
}

}  // namespace

extern "C" {

void rsgpu_options_default(rsgpu_options *out) {
  if (!out) return;
  std::memset(out, 0, sizeof(*out));
  out->inversion_cache = 1;
  out->codec_family = RSGPU_FAMILY_CLASSIC;
  out->leopard_mode = RSGPU_LEOPARD_DISABLED;
  out->matrix_mode = RSGPU_MATRIX_VANDERMONDE;
}

int32_t rsgpu_codec_new(size_t k, size_t m, const rsgpu_options *opts, rsgpu_codec **out) {
  return new_codec(k, m, opts, nullptr, RSGPU_FIELD_GF8, out);
}

int32_t rsgpu_codec_with_custom_matrix(size_t k, size_t m, const uint8_t *rows, const rsgpu_options *opts,
                                       rsgpu_codec **out) {
  if (!rows) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
  return new_codec(k, m, opts, rows, RSGPU_FIELD_GF8, out);
}

int32_t rsgpu_codec_new_gf16(size_t k, size_t m, rsgpu_codec **out) {
  return new_codec(k, m, nullptr, nullptr, RSGPU_FIELD_GF16_TOWER, out);
}

int32_t rsgpu_codec_gf16_with_custom_matrix(size_t k, size_t m, const uint8_t *rows, rsgpu_codec **out) {
  if (!rows) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
  return new_codec(k, m, nullptr, rows, RSGPU_FIELD_GF16_TOWER, out);
}

void rsgpu_codec_free(rsgpu_codec *h) {
  if (!h) return;
  if (h->io[0]) {
    cudaStreamSynchronize(h->io[0]);
    cudaStreamSynchronize(h->io[1]);
    cudaStreamDestroy(h->io[0]);
    cudaStreamDestroy(h->io[1]);
  }
  delete h;
}

size_t rsgpu_data_shard_count(const rsgpu_codec *h) { return h ? h->c.k : 0; }
size_t rsgpu_parity_shard_count(const rsgpu_codec *h) { return h ? h->c.m : 0; }
size_t rsgpu_total_shard_count(const rsgpu_codec *h) { return h ? h->c.k + h->c.m : 0; }
int32_t rsgpu_codec_family(const rsgpu_codec *h) { return h ? h->c.family : -1; }

int32_t rsgpu_encoding_matrix(const rsgpu_codec *h, uint8_t *out, size_t out_len) {
  if (!h || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  const Codec &c = h->c;
  if (c.family != RSGPU_FAMILY_CLASSIC) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  if (c.field == RSGPU_FIELD_GF16_TOWER) {
    if (out_len < c.tmatrix.size() * 2) return RSGPU_ERR_INVALID_ARGUMENT;
    for (size_t i = 0; i < c.tmatrix.size(); ++i) {
      out[2 * i] = c.tmatrix[i].x;
      out[2 * i + 1] = c.tmatrix[i].c;
    }
    return RSGPU_OK;
  }
  if (out_len < c.matrix.size()) return RSGPU_ERR_INVALID_ARGUMENT;
  std::memcpy(out, c.matrix.data(), c.matrix.size());
  return RSGPU_OK;
}

int32_t rsgpu_encode(const rsgpu_codec *hc, uint8_t *const *shards, const size_t *lens, size_t n, int32_t mem,
                     void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !shards || !lens) return RSGPU_ERR_INVALID_ARGUMENT;
  size_t len = 0;
  int rc = h->c.check_all(lens, n, &len);
  if (rc) return rc;
  if ((rc = check_family_len(h->c, len))) return rc;
  if (mem == RSGPU_MEM_DEVICE) return do_encode(h->c, 1, shards, len, S(stream));
  return run_host(h, OP_ENCODE, 1, shards, nullptr, len, 0, nullptr, 0, nullptr, stream);
}

int32_t rsgpu_encode_sep(const rsgpu_codec *hc, const uint8_t *const *data, const size_t *dl, size_t nd,
                         uint8_t *const *parity, const size_t *pl, size_t np, int32_t mem, void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !data || !dl || !parity || !pl) return RSGPU_ERR_INVALID_ARGUMENT;
  const Codec &c = h->c;
  // check_piece_count!(data), (parity), then check_slices!(multi, multi)
  // (src/core/encode.rs:955-958).
  if (nd < c.k) return RSGPU_ERR_TOO_FEW_DATA_SHARDS;
  if (nd > c.k) return RSGPU_ERR_TOO_MANY_DATA_SHARDS;
  if (np < c.m) return RSGPU_ERR_TOO_FEW_PARITY_SHARDS;
  if (np > c.m) return RSGPU_ERR_TOO_MANY_PARITY_SHARDS;
  if (dl[0] == 0) return RSGPU_ERR_EMPTY_SHARD;
  for (size_t i = 0; i < nd; ++i)
    if (dl[i] != dl[0]) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  if (pl[0] == 0) return RSGPU_ERR_EMPTY_SHARD;
  for (size_t i = 0; i < np; ++i)
    if (pl[i] != pl[0]) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  if (dl[0] != pl[0]) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  int rc = check_family_len(c, dl[0]);
  if (rc) return rc;
  std::vector<uint8_t *> all(c.k + c.m);
  for (size_t i = 0; i < c.k; ++i) all[i] = const_cast<uint8_t *>(data[i]);
  for (size_t i = 0; i < c.m; ++i) all[c.k + i] = parity[i];
  if (mem == RSGPU_MEM_DEVICE) return do_encode(h->c, 1, all.data(), dl[0], S(stream));
  return run_host(h, OP_ENCODE, 1, all.data(), nullptr, dl[0], 0, nullptr, 0, nullptr, stream);
}

int32_t rsgpu_verify(const rsgpu_codec *hc, const uint8_t *const *shards, const size_t *lens, size_t n,
                     int32_t *ok, int32_t mem, void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !shards || !lens || !ok) return RSGPU_ERR_INVALID_ARGUMENT;
  size_t len = 0;
  int rc = h->c.check_all(lens, n, &len);
  if (rc) return rc;
  if ((rc = check_family_len(h->c, len))) return rc;
  uint8_t flag = 0;
  if (mem == RSGPU_MEM_DEVICE)
    rc = do_verify(h->c, 1, shards, len, &flag, S(stream));
  else
    rc = run_host(h, OP_VERIFY, 1, const_cast<uint8_t *const *>(shards), nullptr, len, 0, nullptr, 0, &flag, stream);
  if (rc == RSGPU_OK) *ok = flag;
  return rc;
}

int32_t rsgpu_verify_ws_new(const rsgpu_codec *h, size_t shard_len, rsgpu_verify_ws **out) {
  if (!h || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  rsgpu_verify_ws *w = new (std::nothrow) rsgpu_verify_ws();
  if (!w) return RSGPU_ERR_OUT_OF_MEMORY;
  w->shard_len = shard_len;
  *out = w;
  return RSGPU_OK;
}

void rsgpu_verify_ws_free(rsgpu_verify_ws *ws) { delete ws; }

int32_t rsgpu_verify_with_workspace(const rsgpu_codec *h, const uint8_t *const *shards, const size_t *lens, size_t n,
                                    rsgpu_verify_ws *ws, int32_t *ok, int32_t mem, void *stream) {
  if (!ws) return RSGPU_ERR_INVALID_ARGUMENT;
  // The workspace adapts to the call's shard length, as VerifyWorkspace::prepare does.
  int rc = rsgpu_verify(h, shards, lens, n, ok, mem, stream);
  if (rc == RSGPU_OK) ws->shard_len = lens[0];
  return rc;
}

int32_t rsgpu_verify_with_buffer(const rsgpu_codec *hc, const uint8_t *const *shards, const size_t *lens, size_t n,
                                 uint8_t *const *buffer, const size_t *blens, size_t nb, int32_t *ok, int32_t mem,
                                 void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !shards || !lens || !ok || !buffer || !blens) return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = h->c;
  const size_t total = c.k + c.m;
  // check_piece_count!(all), check_piece_count!(parity_buf),
  // check_slices!(multi => slices, multi => buffer) (src/core/verify.rs:161-163).
  if (n < total) return RSGPU_ERR_TOO_FEW_SHARDS;
  if (n > total) return RSGPU_ERR_TOO_MANY_SHARDS;
  if (nb < c.m) return RSGPU_ERR_TOO_FEW_BUFFER_SHARDS;
  if (nb > c.m) return RSGPU_ERR_TOO_MANY_BUFFER_SHARDS;
  size_t len = 0;
  int rc = c.check_all(lens, n, &len);
  if (rc) return rc;
  if (blens[0] == 0) return RSGPU_ERR_EMPTY_SHARD;
  for (size_t i = 0; i < nb; ++i)
    if (blens[i] != blens[0]) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  if (blens[0] != len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  if ((rc = check_family_len(c, len))) return rc;
  // Device pointers: k data, m stored parity, m buffers.
  auto run = [&](uint8_t *const *d, cudaStream_t s) -> int {
    uint8_t flag = 0;
    int r;
    if (c.family == RSGPU_FAMILY_CLASSIC && c.field == RSGPU_FIELD_GF8) {
      r = c.verify_with_buffer_dev(d, len, &flag, s);  // one K1 pass: compare and store
    } else {
      // Leopard and the tower field: encode into the buffers, then compare
      // them with the stored parity (src/core/verify.rs:35-57).
      std::vector<uint8_t *> enc(d, d + c.k);
      enc.insert(enc.end(), d + total, d + total + c.m);
      r = do_encode(c, 1, enc.data(), len, s);
      std::vector<rsgpu::PairOp> pairs(c.m);
      for (size_t i = 0; i < c.m; ++i) pairs[i] = {d[total + i], d[c.k + i], len};
      if (r == RSGPU_OK) r = rsgpu::run_pairs(pairs, rsgpu::PAIR_COMPARE, &flag, s);
    }
    if (r == RSGPU_OK) *ok = flag;
    return r;
  };
  std::vector<uint8_t *> all(total + c.m);
  for (size_t i = 0; i < total; ++i) all[i] = const_cast<uint8_t *>(shards[i]);
  for (size_t i = 0; i < c.m; ++i) all[total + i] = buffer[i];
  if (mem == RSGPU_MEM_DEVICE) return run(all.data(), S(stream));
  std::vector<uint8_t> in(total + c.m, 0), out(total + c.m, 0);
  std::vector<size_t> hl(total + c.m, len);
  for (size_t i = 0; i < total; ++i) in[i] = 1;
  for (size_t i = total; i < total + c.m; ++i) out[i] = 1;
  return run_host_single(h, total + c.m, all.data(), hl.data(), in, out, stream, run);
}

int32_t rsgpu_decode_idx(const rsgpu_codec *hc, uint8_t *const *dst, const size_t *dst_lens, size_t n_dst,
                         const uint8_t *expect, size_t n_expect, const uint8_t *const *input,
                         const size_t *input_lens, size_t n_input, int32_t mem, void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || (!dst && n_dst) || (!dst_lens && n_dst) || (!input && n_input) || (!input_lens && n_input))
    return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = h->c;
  const size_t total = c.k + c.m;
  // src/galois_8/policy.rs:543-700, checks in the reference's order.
  if (c.family != RSGPU_FAMILY_CLASSIC || c.field != RSGPU_FIELD_GF8) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  for (size_t cnt : {n_dst, n_input}) {
    if (cnt < total) return RSGPU_ERR_TOO_FEW_SHARDS;
    if (cnt > total) return RSGPU_ERR_TOO_MANY_SHARDS;
  }
  std::vector<uint8_t> in(2 * total, 0), out(2 * total, 0);
  std::vector<size_t> hl(2 * total, 0);
  std::vector<uint8_t *> host(2 * total, nullptr);  // dst[0..total), input[total..2 total)
  for (size_t i = 0; i < total; ++i) {
    host[i] = dst[i];
    hl[i] = dst[i] ? dst_lens[i] : 0;
    in[i] = out[i] = dst[i] != nullptr;
    host[total + i] = const_cast<uint8_t *>(input[i]);
    hl[total + i] = input[i] ? input_lens[i] : 0;
    in[total + i] = input[i] != nullptr;
  }
  std::function<int(uint8_t *const *, cudaStream_t)> run;
  if (!expect) {
    // Merge mode: validate every pair, then dst[i] ^= input[i].
    for (size_t i = 0; i < total; ++i) {
      if (!input[i]) continue;
      if (!dst[i]) return RSGPU_ERR_TOO_FEW_SHARDS;
      if (dst_lens[i] != input_lens[i]) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
    }
    for (size_t i = 0; i < total; ++i)  // only destinations that receive an input are staged
      if (!input[i]) host[i] = nullptr, in[i] = out[i] = 0;
    run = [&](uint8_t *const *d, cudaStream_t s) {
      std::vector<rsgpu::PairOp> pairs;
      for (size_t i = 0; i < total; ++i)
        if (d[total + i] && input_lens[i]) pairs.push_back({d[total + i], d[i], input_lens[i]});
      return rsgpu::run_pairs(pairs, rsgpu::PAIR_XOR, nullptr, s);
    };
  } else {
    if (n_expect != total) return RSGPU_ERR_INVALID_SHARD_FLAGS;
    std::vector<uint16_t> valid;
    for (size_t i = 0; i < total; ++i)
      if (expect[i]) valid.push_back(uint16_t(i));
    if (valid.size() < c.k) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
    bool have = false;
    size_t len = 0;
    for (size_t i = 0; i < total && !have; ++i)
      if (input[i]) len = input_lens[i], have = true;
    for (size_t i = 0; i < total && !have; ++i)
      if (dst[i]) len = dst_lens[i], have = true;
    if (!have) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
    for (size_t i = 0; i < total; ++i)
      if (input[i] && input_lens[i] != len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
    for (size_t i = 0; i < total; ++i)
      if (dst[i] && dst_lens[i] != len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
    std::vector<uint16_t> outs, cols;
    for (size_t i = 0; i < total; ++i)
      if (dst[i]) outs.push_back(uint16_t(i));
    if (outs.empty()) return RSGPU_OK;
    for (size_t j = 0; j < c.k; ++j)
      if (input[valid[j]]) cols.push_back(uint16_t(j));
    if (cols.empty()) return RSGPU_OK;
    // get_data_decode_matrix takes exactly k selected inputs
    // (src/core/reconstruct.rs:1176-1183).
    if (valid.size() != c.k) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
    if (len == 0) return RSGPU_OK;
    run = [&c, valid, outs, cols, len, total](uint8_t *const *d, cudaStream_t s) {
      return c.decode_idx_dev(valid, outs, cols, d, d + total, len, s);
    };
    // Only the inputs that take part are staged.
    for (size_t i = 0; i < total; ++i) in[total + i] = 0, host[total + i] = nullptr;
    for (uint16_t j : cols) {
      const size_t i = valid[j];
      host[total + i] = const_cast<uint8_t *>(input[i]);
      in[total + i] = 1;
    }
  }
  if (mem == RSGPU_MEM_DEVICE) {
    std::vector<uint8_t *> d(2 * total, nullptr);
    for (size_t i = 0; i < total; ++i) {
      d[i] = dst[i];
      d[total + i] = const_cast<uint8_t *>(input[i]);
    }
    return run(d.data(), S(stream));
  }
  return run_host_single(h, 2 * total, host.data(), hl.data(), in, out, stream, run);
}

int32_t rsgpu_reconstruct(const rsgpu_codec *hc, uint8_t *const *shards, const size_t *lens, const uint8_t *present,
                          size_t n, int32_t goal, const uint8_t *required, size_t n_required, int32_t mem,
                          void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !shards || !lens || !present) return RSGPU_ERR_INVALID_ARGUMENT;
  if (goal == RSGPU_GOAL_REQUIRED && !required) return RSGPU_ERR_INVALID_SHARD_FLAGS;
  size_t len = 0;
  int rc = check_reconstruct(h->c, lens, present, n, goal, required, n_required, &len);
  if (rc || len == 0) return rc;
  if (mem == RSGPU_MEM_DEVICE) return do_reconstruct(h->c, 1, shards, present, len, goal, required, n_required, S(stream));
  return run_host(h, OP_RECONSTRUCT, 1, shards, present, len, goal, required, n_required, nullptr, stream);
}

int32_t rsgpu_prepare_reconstruct_ws(const rsgpu_codec *hc, const uint8_t *present, size_t n, size_t shard_len,
                                     int32_t goal, const uint8_t *required, size_t n_required,
                                     rsgpu_reconstruct_ws **out) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !present || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  Codec &c = h->c;
  const size_t total = c.k + c.m;
  // prepare_reconstruct_some_workspace checks the mask length first, then
  // prepare_reconstruct_workspace_with_goal: piece count, family, shard
  // lengths, then the plan (src/core/reconstruct.rs:586-616,
  // src/core/recovery_plan.rs:300-326, 413-517).
  if (goal == RSGPU_GOAL_REQUIRED && (!required || (n_required != c.k && n_required != total)))
    return RSGPU_ERR_INVALID_SHARD_FLAGS;
  if (n < total) return RSGPU_ERR_TOO_FEW_SHARDS;
  if (n > total) return RSGPU_ERR_TOO_MANY_SHARDS;
  if (c.family != RSGPU_FAMILY_CLASSIC) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  size_t np = 0;
  for (size_t i = 0; i < n; ++i) np += present[i] ? 1 : 0;
  if (np && shard_len == 0) return RSGPU_ERR_EMPTY_SHARD;
  if (np < c.k) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
  int rc = check_family_len(c, shard_len);
  if (rc) return rc;
  std::unique_ptr<rsgpu_reconstruct_ws> w(new (std::nothrow) rsgpu_reconstruct_ws());
  if (!w) return RSGPU_ERR_OUT_OF_MEMORY;
  w->k = c.k;
  w->m = c.m;
  size_t flen = 0;
  if ((rc = rsgpu_format_id(h, nullptr, 0, &flen))) return rc;
  w->format.resize(flen);
  if ((rc = rsgpu_format_id(h, w->format.data(), flen, &flen))) return rc;
  w->present.assign(present, present + n);
  w->shard_len = shard_len;
  w->goal = goal;
  if (goal == RSGPU_GOAL_REQUIRED) w->required.assign(required, required + n_required);
  for (size_t i = 0; i < n; ++i) {
    if (present[i]) continue;
    bool t = goal == RSGPU_GOAL_ALL || (goal == RSGPU_GOAL_DATA && i < c.k) ||
             (goal == RSGPU_GOAL_REQUIRED && i < n_required && required[i]);
    if (t) w->targets.push_back(i);
  }
  if (c.field == RSGPU_FIELD_GF8 && !w->targets.empty()) {
    // The plan's decode tables, built (K3) or taken from the cache now and
    // copied into memory the workspace owns: a singular custom matrix fails
    // here, like the reference's eager inverse.
    rsgpu::ClassicPlan p;
    if ((rc = c.plan_classic(present, goal, required, n_required, p))) return rc;
    std::vector<const rsgpu::ClassicPlan *> pp{&p};
    std::vector<const uint32_t *> tbls;
    std::lock_guard<std::mutex> g(h->io_mu);
    if ((rc = ensure_io(h))) return rc;
    if ((rc = c.decode_tables_copy(pp, tbls, &w->tbl, h->io[0]))) return rc;
    w->survivors = p.survivors;
  }
  *out = w.release();
  return RSGPU_OK;
}

void rsgpu_reconstruct_ws_free(rsgpu_reconstruct_ws *ws) { delete ws; }

size_t rsgpu_reconstruct_ws_targets(const rsgpu_reconstruct_ws *ws, size_t *out, size_t cap) {
  if (!ws) return 0;
  for (size_t i = 0; i < ws->targets.size() && i < cap && out; ++i) out[i] = ws->targets[i];
  return ws->targets.size();
}

int32_t rsgpu_reconstruct_with_ws(const rsgpu_codec *hc, rsgpu_reconstruct_ws *ws, uint8_t *const *shards,
                                  const size_t *lens, const uint8_t *present, size_t n, int32_t mem, void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !ws || !present || !lens || !shards) return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = h->c;
  const size_t total = c.k + c.m;
  // validate_reconstruct_workspace (src/core/reconstruct.rs:702-726): piece
  // count, family, the workspace's shape and format, then the layout
  // (src/core/recovery_plan.rs:390-411): present lengths, the same missing
  // pattern, the same length.
  if (n < total) return RSGPU_ERR_TOO_FEW_SHARDS;
  if (n > total) return RSGPU_ERR_TOO_MANY_SHARDS;
  if (c.family != RSGPU_FAMILY_CLASSIC) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  if (ws->k < c.k) return RSGPU_ERR_TOO_FEW_DATA_SHARDS;
  if (ws->k > c.k) return RSGPU_ERR_TOO_MANY_DATA_SHARDS;
  if (ws->m < c.m) return RSGPU_ERR_TOO_FEW_PARITY_SHARDS;
  if (ws->m > c.m) return RSGPU_ERR_TOO_MANY_PARITY_SHARDS;
  size_t flen = 0;
  int rc = rsgpu_format_id(h, nullptr, 0, &flen);
  if (rc) return rc;
  std::vector<uint8_t> fmt(flen);
  if ((rc = rsgpu_format_id(h, fmt.data(), flen, &flen))) return rc;
  if (fmt != ws->format) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
  size_t len = 0;
  bool same = true;
  for (size_t i = 0; i < n; ++i) {
    if (present[i]) {
      if (lens[i] == 0) return RSGPU_ERR_EMPTY_SHARD;
      if (len && lens[i] != len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
      len = lens[i];
    }
    same &= (present[i] != 0) == (ws->present[i] != 0);
  }
  if (!same) return RSGPU_ERR_INVALID_SHARD_FLAGS;
  if (len != ws->shard_len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  for (size_t t : ws->targets)
    if (lens[t] < len) return RSGPU_ERR_INCORRECT_SHARD_SIZE;
  if (ws->targets.empty()) return RSGPU_OK;
  if (!ws->tbl)  // tower field: the per-call path over the same plan
    return rsgpu_reconstruct(h, shards, lens, present, n, ws->goal,
                             ws->required.empty() ? nullptr : ws->required.data(), ws->required.size(), mem, stream);
  // GF(2^8): one K1 job over the plan's survivors and targets with the
  // workspace's own tables.
  auto run = [&](uint8_t *const *d, cudaStream_t s) {
    std::vector<rsgpu::JobDesc> jobs(1);
    jobs[0].n_in = uint16_t(c.k);
    jobs[0].n_out = uint16_t(ws->targets.size());
    jobs[0].tbl = ws->tbl;
    std::vector<const uint8_t *> ptrs;
    for (uint16_t sv : ws->survivors) ptrs.push_back(d[sv]);
    for (size_t t : ws->targets) ptrs.push_back(d[t]);
    return c.apply_jobs(jobs, ptrs, len, s);
  };
  if (mem == RSGPU_MEM_DEVICE) return run(shards, S(stream));
  std::vector<uint8_t> in(n, 0), out(n, 0);
  std::vector<uint8_t *> host(n, nullptr);
  std::vector<size_t> hl(n, len);
  for (uint16_t sv : ws->survivors) host[sv] = shards[sv], in[sv] = 1;
  for (size_t t : ws->targets) host[t] = shards[t], out[t] = 1;
  return run_host_single(h, n, host.data(), hl.data(), in, out, stream, run);
}

int32_t rsgpu_encode_batch(const rsgpu_codec *hc, size_t n_stripes, uint8_t *const *ptrs, size_t len, int32_t mem,
                           void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || (!ptrs && n_stripes)) return RSGPU_ERR_INVALID_ARGUMENT;
  if (len == 0) return RSGPU_ERR_EMPTY_SHARD;
  int rc = check_family_len(h->c, len);
  if (rc || n_stripes == 0) return rc;
  if (mem == RSGPU_MEM_DEVICE) return do_encode(h->c, n_stripes, ptrs, len, S(stream));
  return run_host(h, OP_ENCODE, n_stripes, ptrs, nullptr, len, 0, nullptr, 0, nullptr, stream);
}

int32_t rsgpu_reconstruct_batch(const rsgpu_codec *hc, size_t n_stripes, uint8_t *const *ptrs,
                                const uint8_t *present, size_t len, int32_t goal, int32_t mem, void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || (!ptrs && n_stripes) || (!present && n_stripes)) return RSGPU_ERR_INVALID_ARGUMENT;
  if (goal == RSGPU_GOAL_REQUIRED) return RSGPU_ERR_INVALID_SHARD_FLAGS;
  if (len == 0) return RSGPU_ERR_EMPTY_SHARD;
  int rc = check_family_len(h->c, len);
  if (rc || n_stripes == 0) return rc;
  const size_t total = h->c.k + h->c.m;
  for (size_t s = 0; s < n_stripes; ++s) {
    size_t np = 0;
    for (size_t i = 0; i < total; ++i) np += present[s * total + i] ? 1 : 0;
    if (np < h->c.k) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
  }
  if (mem == RSGPU_MEM_DEVICE) return do_reconstruct(h->c, n_stripes, ptrs, present, len, goal, nullptr, 0, S(stream));
  return run_host(h, OP_RECONSTRUCT, n_stripes, ptrs, present, len, goal, nullptr, 0, nullptr, stream);
}

int32_t rsgpu_verify_batch(const rsgpu_codec *hc, size_t n_stripes, const uint8_t *const *ptrs, size_t len,
                           uint8_t *ok, int32_t mem, void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || (!ptrs && n_stripes) || (!ok && n_stripes)) return RSGPU_ERR_INVALID_ARGUMENT;
  if (len == 0) return RSGPU_ERR_EMPTY_SHARD;
  int rc = check_family_len(h->c, len);
  if (rc || n_stripes == 0) return rc;
  if (mem == RSGPU_MEM_DEVICE) return do_verify(h->c, n_stripes, ptrs, len, ok, S(stream));
  return run_host(h, OP_VERIFY, n_stripes, const_cast<uint8_t *const *>(ptrs), nullptr, len, 0, nullptr, 0, ok,
                  stream);
}

int32_t rsgpu_batch_prepare(const rsgpu_codec *hc, int32_t op, size_t n_stripes, uint8_t *const *ptrs,
                            const uint8_t *present, size_t len, int32_t goal, rsgpu_batch **out) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !out || (!ptrs && n_stripes)) return RSGPU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (op < RSGPU_OP_ENCODE || op > RSGPU_OP_VERIFY) return RSGPU_ERR_INVALID_ARGUMENT;
  if (op == RSGPU_OP_RECONSTRUCT && (!present || goal == RSGPU_GOAL_REQUIRED)) return RSGPU_ERR_INVALID_SHARD_FLAGS;
  if (len == 0) return RSGPU_ERR_EMPTY_SHARD;
  Codec &c = h->c;
  int rc = check_family_len(c, len);
  if (rc) return rc;
  const size_t total = c.k + c.m;
  if (op == RSGPU_OP_RECONSTRUCT)
    for (size_t s = 0; s < n_stripes; ++s) {
      size_t np = 0;
      for (size_t i = 0; i < total; ++i) np += present[s * total + i] ? 1 : 0;
      if (np < c.k) return RSGPU_ERR_TOO_FEW_SHARDS_PRESENT;
    }
  std::unique_ptr<rsgpu_batch> b(new (std::nothrow) rsgpu_batch());
  if (!b) return RSGPU_ERR_OUT_OF_MEMORY;
  b->codec = h;
  b->op = op;
  b->n_stripes = n_stripes;
  if (op == RSGPU_OP_VERIFY) {
    RS_CUDA(cudaMalloc(reinterpret_cast<void **>(&b->flags), std::max<size_t>(n_stripes, 1) * 4));
    RS_CUDA(cudaMemset(b->flags, 0, std::max<size_t>(n_stripes, 1) * 4));
  }
  if (c.family != RSGPU_FAMILY_CLASSIC || c.field != RSGPU_FIELD_GF8) {
    rc = rsgpu::prepare_other(c, op, n_stripes, ptrs, present, len, goal, b->flags, b->leo);
  } else {
    std::vector<rsgpu::JobDesc> jobs;
    std::vector<const uint8_t *> dptrs;
    if (op == RSGPU_OP_RECONSTRUCT) {
      rc = c.reconstruct_jobs(n_stripes, ptrs, present, goal, nullptr, 0, jobs, dptrs, nullptr, &b->owned_tables);
      if (rc == RSGPU_OK) rc = rsgpu::cuda_status(cudaDeviceSynchronize());
    } else {
      rc = c.encode_jobs(n_stripes, ptrs, jobs, dptrs, op == RSGPU_OP_VERIFY);
    }
    if (rc == RSGPU_OK) rc = b->apply.build(jobs, dptrs, len, op == RSGPU_OP_VERIFY, b->flags, nullptr, true);
    b->apply.args.stall = c.d_status;
  }
  if (rc) return rc;
  *out = b.release();
  return RSGPU_OK;
}

int32_t rsgpu_batch_launch(rsgpu_batch *b, void *stream) {
  if (!b) return RSGPU_ERR_INVALID_ARGUMENT;
  if (b->flags) RS_CUDA(cudaMemsetAsync(b->flags, 0, std::max<size_t>(b->n_stripes, 1) * 4, S(stream)));
  if (b->leo) return rsgpu::leo_launch(*b->leo, S(stream));
  return b->apply.launch(S(stream));
}

int32_t rsgpu_batch_verify_result(rsgpu_batch *b, uint8_t *ok, void *stream) {
  if (!b || !ok || b->op != RSGPU_OP_VERIFY) return RSGPU_ERR_INVALID_ARGUMENT;
  std::vector<uint32_t> f(b->n_stripes);
  RS_CUDA(cudaMemcpyAsync(f.data(), b->flags, b->n_stripes * 4, cudaMemcpyDeviceToHost, S(stream)));
  RS_CUDA(cudaStreamSynchronize(S(stream)));
  for (size_t i = 0; i < b->n_stripes; ++i) ok[i] = f[i] ? 0 : 1;
  return RSGPU_OK;
}

uint32_t rsgpu_batch_kernel_count(const rsgpu_batch *b) {
  if (!b) return 0;
  if (b->leo) return rsgpu::leo_kernel_count(*b->leo);
  return uint32_t((b->apply.args.any_vec ? 1 : 0) + (b->apply.max_tail ? 1 : 0));
}

void rsgpu_batch_free(rsgpu_batch *b) { delete b; }

int32_t rsgpu_get_cache_stats(const rsgpu_codec *h, rsgpu_cache_stats *out) {
  if (!h || !out) return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = const_cast<rsgpu_codec *>(h)->c;
  if (c.family != RSGPU_FAMILY_CLASSIC)
    rsgpu::leopard_cache_stats(c, out);  // the error-locator cache
  else
    c.stats(out);
  return RSGPU_OK;
}

int32_t rsgpu_leopard_reconstruct_noalloc(const rsgpu_codec *hc, uint8_t *const *shards, const size_t *lens,
                                          const uint8_t *present, size_t n, void *stream) {
  rsgpu_codec *h = const_cast<rsgpu_codec *>(hc);
  if (!h || !shards || !lens || !present) return RSGPU_ERR_INVALID_ARGUMENT;
  Codec &c = h->c;
  if (c.family == RSGPU_FAMILY_CLASSIC) return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY;
  size_t len = 0;
  int rc = check_reconstruct(c, lens, present, n, RSGPU_GOAL_ALL, nullptr, 0, &len);
  if (rc || len == 0) return rc;
  return rsgpu::leopard_reconstruct_noalloc(c, shards, present, len, S(stream));
}

uint64_t rsgpu_kernel_launch_count(void) { return rsgpu::launch_counter(); }

const char *rsgpu_error_string(int32_t code) {
  switch (code) {
    case RSGPU_OK: return "ok";
    case RSGPU_ERR_TOO_FEW_SHARDS: return "The number of provided shards is smaller than the one in codec";
    case RSGPU_ERR_TOO_MANY_SHARDS: return "The number of provided shards is greater than the one in codec";
    case RSGPU_ERR_TOO_FEW_DATA_SHARDS: return "The number of provided data shards is smaller than the one in codec";
    case RSGPU_ERR_TOO_MANY_DATA_SHARDS: return "The number of provided data shards is greater than the one in codec";
    case RSGPU_ERR_TOO_FEW_PARITY_SHARDS: return "The number of provided parity shards is smaller than the one in codec";
    case RSGPU_ERR_TOO_MANY_PARITY_SHARDS: return "The number of provided parity shards is greater than the one in codec";
    case RSGPU_ERR_TOO_FEW_BUFFER_SHARDS: return "The number of provided buffer shards is smaller than the number of parity shards in codec";
    case RSGPU_ERR_TOO_MANY_BUFFER_SHARDS: return "The number of provided buffer shards is greater than the number of parity shards in codec";
    case RSGPU_ERR_INCORRECT_SHARD_SIZE: return "At least one of the provided shards is not of the correct size";
    case RSGPU_ERR_TOO_FEW_SHARDS_PRESENT: return "The number of present shards is smaller than the number of data shards required for reconstruction";
    case RSGPU_ERR_EMPTY_SHARD: return "The first shard provided is of zero length";
    case RSGPU_ERR_INVALID_SHARD_FLAGS: return "The number of flags does not match the total number of shards";
    case RSGPU_ERR_INVALID_INDEX: return "The data shard index provided is greater or equal to the number of data shards in codec";
    case RSGPU_ERR_INVALID_CUSTOM_MATRIX: return "The encoding matrix is invalid, missing, or incompatible with the reconstruction workspace";
    case RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY: return "The selected codec family is not supported for this field or configuration";
    case RSGPU_ERR_UNSUPPORTED_LEOPARD_PROTOTYPE: return "The selected Leopard codec family is only available as a prototype skeleton in this build";
    case RSGPU_ERR_CUDA: return "CUDA runtime error";
    case RSGPU_ERR_OUT_OF_MEMORY: return "device memory exhausted";
    case RSGPU_ERR_INVALID_ARGUMENT: return "invalid argument (null pointer or undersized output)";
    case RSGPU_ERR_DEVICE_TIMEOUT: return "a bounded device wait expired";
    case RSGPU_ERR_NO_DEVICE: return "no CUDA device available";
    case RSGPU_ERR_SCRATCH_LIMIT: return "the code is wider than the no-allocation entry point's static buffers allow";
    case RSGPU_ERR_STREAM_IO: return "a stream read or write callback failed";
    default: return "unknown error";
  }
}

const char *rsgpu_version(void) { return "rsgpu 0.1.0 sm_100a"; }

}  // extern "C"
