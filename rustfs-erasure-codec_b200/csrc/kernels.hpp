// kernels.hpp -- launch interfaces of the sm_100a kernels (host <-> device).
#pragma once

#include <cuda_runtime.h>

#include "common.hpp"

namespace rsgpu {

// K1 arguments (k_classic.cu).
struct ApplyArgs {
  const JobDesc *jobs;          // device, n_jobs
  const uint8_t *const *ptrs;   // device pointer table
  uint32_t *flags;              // device verify flags (may be null for writes)
  uint64_t len;                 // bytes per shard (same for every job)
  uint32_t n_jobs;
  uint32_t max_out;             // largest n_out over the jobs
  int any_vec;                  // some job has vec_len > 0
  int accumulate;               // outputs ^= products (incremental parity update)
  uint32_t *stall;              // device status word: a bounded wait of the TMA-staged tile ran out (may be null)
  int tbl_stage;                // jobs carry different tables: the TMA-staged tile copies them with the data
};
cudaError_t launch_apply(const ApplyArgs &a, bool verify, uint64_t max_tail, cudaStream_t s);
// K1 tile for launches of at most 4 outputs: 0 (default) TMA-staged, 1 the
// register-path tile, 2 / 3 other TMA ring shapes; RSGPU_APPLY_VARIANT picks
// one for measurements.
int &apply_variant();

// K3: one erasure pattern.  Indices fit a byte because classic codecs have at
// most 256 shards.
struct DecodeTask {
  uint8_t survivors[256];  // first k present shard indices, ascending
  uint8_t targets[256];    // requested missing indices: data first, then parity
  uint32_t n_out;
  uint32_t needs_inverse;  // some missing data shard feeds an output
  uint32_t pad;
  uint32_t *tbl_out;       // device destination of the packed tables
};
struct DecodeTableArgs {
  const DecodeTask *tasks;  // device
  const uint8_t *matrix;    // device, (k+m) x k encoding matrix
  const uint8_t *gf_log;    // device, 256
  const uint8_t *gf_exp;    // device, >= 255
  int *status;              // device, per task: 0 ok, 1 singular
  int k;
};
cudaError_t launch_decode_tables(const DecodeTableArgs &a, int n_tasks, int max_out, cudaStream_t s);

// Bytewise work over pairs of equally long buffers (device array `pairs`):
// PAIR_COMPARE ORs 1 into *flag when some pair differs (the comparison step
// of verify_with_buffer for codecs whose parity comes from a separate encode
// launch); PAIR_XOR sets b ^= a (decode_idx merge mode).
struct PairOp {
  const uint8_t *a;
  uint8_t *b;
  uint64_t len;
};
enum { PAIR_COMPARE = 0, PAIR_XOR = 1 };
cudaError_t launch_pairs(const PairOp *pairs, uint32_t n, uint64_t max_len, int mode, uint32_t *flag,
                         cudaStream_t s);

// Packed tables of a subset of a packed table's input columns: out holds, for
// every group of 4 outputs, the tables of inputs cols[0..n_sel) of `full`
// (groups x k_full inputs), in that order (decode_idx over the inputs one
// call supplies).
struct GatherCols {
  uint8_t cols[256];
};
cudaError_t launch_gather_tables(const uint32_t *full, uint32_t *out, const GatherCols &cols, uint32_t groups,
                                 uint32_t k_full, uint32_t n_sel, cudaStream_t s);

}  // namespace rsgpu
