// codec.hpp -- the host runtime behind the C ABI.
//
// A Codec mirrors the reference `ReedSolomon<F>` (src/core/codec.rs): it owns
// the encoding matrix (classic) or the FFT tables (Leopard), validates every
// call with the reference's error precedence before any launch, plans
// reconstruction, keeps decode tables resident in HBM keyed by erasure
// pattern, and drives the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <list>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.hpp"
#include "gf_host.hpp"
#include "kernels.hpp"

namespace rsgpu {

// Result of the classic recovery planner for one erasure pattern
// (src/core/recovery_plan.rs:262-517).
struct ClassicPlan {
  int status = RSGPU_OK;
  bool all_present = false;
  bool needs_inverse = false;
  std::vector<uint16_t> survivors;  // first k present indices
  std::vector<uint16_t> targets;    // requested missing indices, ascending
  size_t n_data_targets = 0;
};

// 256-bit presence / target masks identify a decode-table entry.
struct PatternKey {
  std::array<uint64_t, 4> present{};
  std::array<uint64_t, 4> targets{};
  bool operator==(const PatternKey &o) const { return present == o.present && targets == o.targets; }
};
struct PatternKeyHash {
  size_t operator()(const PatternKey &k) const {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    for (int i = 0; i < 4; ++i) {
      h ^= k.present[i] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
      h ^= k.targets[i] + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    }
    return size_t(h);
  }
};

struct DecodeEntry {
  uint32_t *tbl = nullptr;  // device, packed tables (block of the table pool)
  std::vector<uint16_t> survivors;
  std::vector<uint16_t> targets;
  std::list<PatternKey>::iterator lru;
};

// Fixed-size device blocks for decode tables, carved from large slabs so a
// cache miss never calls cudaMalloc.
class TablePool {
 public:
  explicit TablePool(size_t block_bytes) : block_(block_bytes) {}
  ~TablePool();
  uint32_t *get();
  void put(uint32_t *p) { free_.push_back(p); }
  size_t block_bytes() const { return block_; }
  size_t slab_bytes() const { return slabs_.size() * kSlab; }

 private:
  static constexpr size_t kSlab = 8u << 20;
  size_t block_;
  std::vector<void *> slabs_;
  std::vector<uint32_t *> free_;
};

struct LeopardState;  // leopard.cu
struct TowerState;    // tower.cu

// A K1 launch whose job and pointer tables live in device memory.  Built once
// and launched any number of times (launch() allocates and synchronizes
// nothing, so it can be captured in a CUDA graph).
struct ApplyLaunch {
  void *d_blob = nullptr;  // JobDesc[n_jobs] followed by the pointer table
  bool owned = false;      // cudaMalloc'd (prepared batch) vs stream-ordered
  ApplyArgs args{};
  uint64_t max_tail = 0;
  bool verify = false;
  int build(std::vector<JobDesc> &jobs, const std::vector<const uint8_t *> &ptrs, size_t len, bool verify,
            uint32_t *flags, cudaStream_t s, bool persistent, bool accumulate = false);
  int launch(cudaStream_t s) const;
  void release(cudaStream_t s);
};

class Codec {
 public:
  size_t k = 0, m = 0;
  int family = RSGPU_FAMILY_CLASSIC;
  int field = RSGPU_FIELD_GF8;
  rsgpu_options opts{};
  int device = 0;
  Mat8 matrix;             // classic GF(2^8): (k+m) x k
  std::vector<T16> tmatrix;  // classic tower field
  // device-resident codec constants
  uint8_t *d_matrix = nullptr;
  uint8_t *d_log = nullptr, *d_exp = nullptr;
  uint32_t *d_enc_tbl = nullptr;  // parity rows packed for K1
  // Set by a K1 launch whose bounded device wait ran out; read and cleared
  // by the next synchronous call (take_device_status).
  uint32_t *d_status = nullptr;
  std::shared_ptr<LeopardState> leo;  // created where the type is complete
  std::shared_ptr<TowerState> tower;

  ~Codec();
  int init_classic(const uint8_t *custom_rows);
  // RSGPU_ERR_DEVICE_TIMEOUT (and clears it) when a launch of this codec
  // recorded a stalled wait; waits for stream s.
  int take_device_status(cudaStream_t s);
  int init_tower(const uint8_t *custom_rows);
  int init_leopard();

  // ---- validation (reference error precedence)
  int check_all(const size_t *lens, size_t n, size_t *shard_len) const;
  int plan_classic(const uint8_t *present, int goal, const uint8_t *required, size_t n_required,
                   ClassicPlan &out) const;

  // ---- operations; pointers are device pointers unless noted
  int encode_dev(size_t n_stripes, uint8_t *const *shards, size_t len, cudaStream_t s);
  // `tbl`: packed parity tables to check against (default: this codec's
  // encode tables d_enc_tbl).
  int verify_dev(size_t n_stripes, const uint8_t *const *shards, size_t len, uint8_t *ok_host, cudaStream_t s,
                 const uint32_t *tbl = nullptr);
  // Verify without waiting: stripe i ORs 1 into flags_dev[i] on a mismatch.
  int verify_dev_async(size_t n_stripes, uint8_t *const *shards, size_t len, uint32_t *flags_dev, cudaStream_t s);
  int reconstruct_dev(size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                      int goal, const uint8_t *required, size_t n_required, cudaStream_t s);
  // verify_with_buffer (src/core/verify.rs:157-176) in one K1 pass: ptrs3
  // holds k data, m stored parity and m buffer pointers; the recomputed
  // parity goes to the buffers and *ok_host says whether it matched.
  int verify_with_buffer_dev(uint8_t *const *ptrs3, size_t len, uint8_t *ok_host, cudaStream_t s);
  // decode_idx (src/galois_8/policy.rs:543-700) after validation: `selected`
  // = the first k expected inputs, `outs` = destination indices, `cols` =
  // positions among `selected` whose input arrived in this call (ascending);
  // dst[outs[o]] ^= sum_j row_o[cols[j]] * input[selected[cols[j]]], rows
  // from the decode-table cache (K3, one entry per m destinations), one
  // accumulating K1 launch.
  int decode_idx_dev(const std::vector<uint16_t> &selected, const std::vector<uint16_t> &outs,
                     const std::vector<uint16_t> &cols, uint8_t *const *dst, const uint8_t *const *input,
                     size_t len, cudaStream_t s);

  // Incremental parity (src/core/encode.rs:890-930, 1048-1120): for one
  // stripe, parity_r (+)= sum_j c[r][j] * in[j] over the given inputs, where
  // c[r][j] = encoding matrix (k + r, cols[j]); `accumulate` adds into the
  // parity instead of overwriting it.  Device pointers.
  int apply_parity_columns(const std::vector<const uint8_t *> &inputs, const std::vector<size_t> &cols,
                           uint8_t *const *parity, size_t len, bool accumulate, cudaStream_t s);

  // K1 over jobs whose `tbl` pointers already point at device tables.
  int apply_jobs(std::vector<JobDesc> &jobs, std::vector<const uint8_t *> &ptrs, size_t len, cudaStream_t s) {
    return run_apply(jobs, ptrs, len, false, nullptr, s);
  }

  // K1 over jobs whose packed tables are given on the host: `tables` is
  // uploaded stream-ordered, job i reads it from word tbl_off[i]; device
  // pointers in `ptrs`.
  int apply_with_tables(std::vector<JobDesc> &jobs, const std::vector<size_t> &tbl_off,
                        std::vector<const uint8_t *> &ptrs, const std::vector<uint32_t> &tables, size_t len,
                        cudaStream_t s);

  // Decode tables for a set of plans, building missing entries on the GPU (K3).
  int decode_tables(const std::vector<const ClassicPlan *> &plans, std::vector<const uint32_t *> &tbls,
                    cudaStream_t s);
  void stats(rsgpu_cache_stats *out);
  // decode_tables for callers that keep the tables beyond the cache's
  // control (prepared and mixed batches): the distinct tables are copied into
  // one new device allocation (*owned, to be cudaFree'd by the caller) before
  // the cache lock is released, so a later eviction cannot recycle them.
  int decode_tables_copy(const std::vector<const ClassicPlan *> &plans, std::vector<const uint32_t *> &tbls,
                         uint32_t **owned, cudaStream_t s);
  // decode_tables under the cache lock, returning the cache's own blocks.
  int decode_tables_shared(const std::vector<const ClassicPlan *> &plans, std::vector<const uint32_t *> &tbls,
                           cudaStream_t s);

 private:
  std::mutex mu_;
  std::unordered_map<PatternKey, DecodeEntry, PatternKeyHash> cache_;
  std::list<PatternKey> lru_;
  std::unique_ptr<TablePool> pool_;
  std::vector<uint32_t *> retire_;  // evicted blocks awaiting a device sync
  rsgpu_cache_stats stats_{};
  size_t capacity_ = 0;
  int run_apply(std::vector<JobDesc> &jobs, std::vector<const uint8_t *> &ptrs, size_t len, bool verify,
                uint32_t *flags_dev, cudaStream_t s, bool accumulate = false);

 public:
  // Job lists for the three classic operations over device pointers.  With
  // `owned`, the decode tables are private copies (see decode_tables_copy).
  int encode_jobs(size_t n_stripes, uint8_t *const *shards, std::vector<JobDesc> &jobs,
                  std::vector<const uint8_t *> &ptrs, bool verify);
  int reconstruct_jobs(size_t n_stripes, uint8_t *const *shards, const uint8_t *present, int goal,
                       const uint8_t *required, size_t n_required, std::vector<JobDesc> &jobs,
                       std::vector<const uint8_t *> &ptrs, cudaStream_t s, uint32_t **owned = nullptr);
};

int cuda_status(cudaError_t e);
// Pair kernel over device buffers (kernels.hpp PairOp): PAIR_COMPARE writes
// *ok_host (waits for s), PAIR_XOR queues b ^= a and returns.
int run_pairs(const std::vector<PairOp> &pairs, int mode, uint8_t *ok_host, cudaStream_t s);

}  // namespace rsgpu
