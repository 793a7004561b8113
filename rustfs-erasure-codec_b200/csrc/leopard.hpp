// leopard.hpp -- family resolution plus the Leopard FFT and tower-field
// classic codecs (device pointers; validation already done by the caller).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "rsgpu.h"

namespace rsgpu {

class Codec;

// A prepared Leopard (or tower-field) batch: device-resident job tables whose
// launch allocates and synchronizes nothing.
struct LeoLaunch;
int prepare_other(Codec &c, int op, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                  int goal, uint32_t *flags, std::shared_ptr<LeoLaunch> &out);
int leo_launch(const LeoLaunch &l, cudaStream_t s);
// A one-shot Leopard reconstruction of n stripes of one codec, shard length
// and goal through the codec's own decode kernel, built on stream s: its job
// blob is allocated on s and freed there, behind the kernel, when the launch
// is destroyed, and building it never waits for the device (a codec's first
// wide decode may grow its work-row slab with cudaMalloc).
// With `scratch` (a device buffer private to stream s, at least
// leo_reconstruct_scratch_bytes(c) bytes) the launch keeps its work rows
// there instead of in the codec's shared slab, so it neither grows that slab
// nor waits for other streams' launches that use it; leo_set_scratch moves it
// to another such buffer before the launch.
int prepare_leo_reconstruct_once(Codec &c, size_t n, uint8_t *const *shards, const uint8_t *present, size_t len,
                                 int goal, cudaStream_t s, void *scratch, std::shared_ptr<LeoLaunch> &out);
size_t leo_reconstruct_scratch_bytes(Codec &c);
void leo_set_scratch(LeoLaunch &l, void *scratch);
int prepare_tower(Codec &c, int op, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                  int goal, uint32_t *flags, std::shared_ptr<LeoLaunch> &out);
uint32_t leo_kernel_count(const LeoLaunch &l);

// src/core/leopard.rs:191-223 (resolve_codec_family) for the byte field.
int resolve_family(int requested, int mode, size_t total, size_t parity);
// src/core/leopard.rs:146-156, 225-270 (validate_leopard_family).
int validate_leopard_family(int family, size_t k, size_t m);

int leopard_encode(Codec &c, size_t n_stripes, uint8_t *const *shards, size_t len, cudaStream_t s);
int leopard_verify(Codec &c, size_t n_stripes, const uint8_t *const *shards, size_t len, uint8_t *ok,
                   cudaStream_t s);
int leopard_reconstruct(Codec &c, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                        int goal, const uint8_t *required, size_t n_required, cudaStream_t s);

// No-allocation Leopard reconstruction (leopard.cu): static device buffers only.
int leopard_reconstruct_noalloc(Codec &c, uint8_t *const *shards, const uint8_t *present, size_t len,
                                cudaStream_t s);

// ---- mixed batches (batch.cu)
struct LeoGeometry {
  int bits;
  uint32_t k, p, m, n, mtrunc, last, mod;
  const uint16_t *skew;
  const uint32_t *bank;   // half-warp layer kernels
  const uint32_t *kbank;  // register-stage kernels
  const uint32_t *sktab;  // kbank's tables of each skew entry
  uint32_t st_ienc, st_fenc, st_idec, st_fdec;  // stage plans (leo_types.hpp)
  uint32_t n_ienc, n_fenc, n_idec, n_fdec;
};
int leopard_geometry(Codec &c, LeoGeometry *g);
// Error locators of n presence patterns (k + m flags each), built on the GPU
// for patterns not in the codec's cache and copied into the caller's device
// buffer `dst` (room for n arrays of the geometry's n lanes); err[i] points at
// pattern i's array there (patterns that repeat share one).  With `ordered`
// the copies are queued on s; otherwise the call waits for them.
int leopard_locators(Codec &c, size_t n, const uint8_t *present, uint16_t *dst, const uint16_t **err,
                     uint32_t *input_count, cudaStream_t s, bool ordered);
// Statistics of the codec's error-locator cache (entries = cached patterns,
// retained_bytes = their device bytes).
void leopard_cache_stats(Codec &c, rsgpu_cache_stats *out);
// Leopard GF(2^8) products: mul[a][b] in the codec field's representation.
const uint8_t (*leopard_mul8())[256];
// The GF(2^8) Leopard encode as a dense m x k matrix over the Leopard field
// (the FFT pipeline is linear, so applying this matrix gives the same bytes).
int leopard_dense_encode(Codec &c, std::vector<uint8_t> &rows);
// The GF(2^8) Leopard reconstruction of one presence pattern as a dense map
// from the present shards (ascending) to the targets (ascending).  The
// reference's decode uses every present shard, and so does this map, so the
// bytes agree on any input, codeword or not.  Maps (with their K1 tables) are
// cached per codec by (pattern, goal), least recently used first out beyond
// 64 MiB; GF(2^8) per-call reconstructs run them through K1.
struct LeoDenseMap {
  std::vector<uint16_t> inputs, targets;
  std::vector<uint8_t> rows;  // targets x inputs
  std::shared_ptr<const std::vector<uint32_t>> packed;  // rows packed for K1 (Leopard multiplication)
};
int leopard_dense_decode(Codec &c, size_t n, const uint8_t *present, int goal, std::vector<LeoDenseMap> &maps,
                         cudaStream_t s);
// Whether one GF(2^8) reconstruct (goal all or data) of this pattern should
// run through the dense map now: its map is cached, or the codec's calls
// have moved 64 MiB under the pattern, this one included (the per-call rule;
// maps of more than 16 targets on shards under 1 MiB stay on the FFT decode).
// Counts this call's bytes towards the pattern's tally.
bool leopard_dense_due(Codec &c, const uint8_t *present, int goal, size_t len);
// Whether the codec's map cache holds this pattern's map.
bool leopard_dense_cached(Codec &c, const uint8_t *present, int goal);
// A GF(2^8) reconstruction's dense map derived and packed on the device, all
// queued on stream s (no host wait): d_img (leopard_dense_inline_bytes bytes)
// holds the unit-vector stripe the pattern's FFT decode runs on, d_tbl
// (packed_table_words(targets, inputs) words) receives the K1 tables.  Both
// buffers must stay allocated until the work queued on s has run.  Returns
// the map's inputs and targets (ascending shard indices); no targets, no work.
size_t leopard_dense_inline_bytes(Codec &c, const uint8_t *present, int goal);
int leopard_dense_inline(Codec &c, const uint8_t *present, int goal, uint8_t *d_img, uint32_t *d_tbl,
                         std::vector<uint16_t> &inputs, std::vector<uint16_t> &targets, cudaStream_t s);

// A map derived off the request path: start queues the FFT decode of the
// pattern's unit vectors on stream s through a caller-owned pinned buffer of
// leopard_dense_derive_bytes bytes (no host wait) and records d.done; once
// d.done has completed, finish packs the map and adds it to the codec's map
// cache.  The codec must outlive the derivation.
struct DenseDerivation {
  Codec *codec = nullptr;
  std::string pattern;  // k + m presence flags
  int goal = 0;
  size_t L = 0, bytes = 0;
  uint8_t *pinned = nullptr;
  uint8_t *dev = nullptr;
  cudaEvent_t done = nullptr;
};
size_t leopard_dense_derive_bytes(Codec &c, const uint8_t *present, int goal);
int leopard_dense_derive_start(Codec &c, const uint8_t *present, int goal, uint8_t *pinned, cudaStream_t s,
                               DenseDerivation &d);
int leopard_dense_derive_finish(DenseDerivation &d);

int tower_encode(Codec &c, size_t n_stripes, uint8_t *const *shards, size_t len, cudaStream_t s);
// Tower-field incremental parity: parity_r (+)= sum_j t[k + r][cols[j]] * inputs[j] (one stripe).
int tower_apply_columns(Codec &c, const std::vector<const uint8_t *> &inputs, const std::vector<size_t> &cols,
                        uint8_t *const *parity, size_t len, bool accumulate, cudaStream_t s);
int tower_verify(Codec &c, size_t n_stripes, const uint8_t *const *shards, size_t len, uint8_t *ok,
                 cudaStream_t s);
int tower_reconstruct(Codec &c, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                      int goal, const uint8_t *required, size_t n_required, cudaStream_t s);

}  // namespace rsgpu
