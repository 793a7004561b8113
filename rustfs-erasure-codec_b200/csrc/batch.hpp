// batch.hpp -- mixed batches (batch.cu) and the plan selector (tuner.cu).
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
struct MixBatch;
struct MixDeleter {
  void operator()(MixBatch *b) const;
};
using MixPtr = std::unique_ptr<MixBatch, MixDeleter>;

// A caller-owned device buffer for the work rows of one-shot batches on one
// stream, reused from batch to batch and grown (in that stream's order) only
// when a batch needs more.  Allocating hundreds of MB per batch instead was
// measured to block the building thread for up to hundreds of milliseconds
// while other streams' kernels ran.  The owner frees `ptr` after the stream's
// work has finished.
struct ScratchSlot {
  void *ptr = nullptr;
  size_t bytes = 0;
};

// A Leopard GF(2^8) rebuild pattern whose dense map is due but not derived
// yet (one-shot batches with `deferred` only).
struct DenseWant {
  const rsgpu_codec *codec;
  std::string pattern;  // k + m presence flags
  int goal;
};

// Prepare a mixed batch; `forced` (optional) gives every op's plan.
// With `ordered`, the batch is a one-shot, stream-ordered batch for that
// stream (no graph): its device memory is allocated and freed in the stream's
// order and building it never synchronizes the device; `scratch` (optional,
// one-shot batches) supplies its work rows.  With `deferred` (one-shot
// batches), a due pattern whose map is not cached runs the FFT decode in this
// batch and is listed in *deferred, for the caller to derive off the request
// path; without it the map is derived before the launch.
int mix_build(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_plan *forced, const rsgpu_mix_options &opt,
              MixPtr &out, cudaStream_t ordered = nullptr, ScratchSlot *scratch = nullptr,
              std::vector<DenseWant> *deferred = nullptr);
// The validation mix_build applies to each operation (reference error
// precedence; shard pointers must be non-null).
int mix_validate(const rsgpu_mix_op &o, int device);
// Device verify flags of a batch (one word per operation, nonzero = mismatch).
const uint32_t *mix_flags(const MixBatch &b);
int mix_launch(MixBatch &b, cudaStream_t s);
int mix_results(MixBatch &b, uint8_t *ok, cudaStream_t s);
const rsgpu_mix_info &mix_info(const MixBatch &b);
const std::vector<rsgpu_plan> &mix_plans(const MixBatch &b);

bool mix_plan_valid(const Codec &c, int op, const rsgpu_plan &p);
rsgpu_plan mix_default_plan(Codec &c, int op, size_t len);

// True when the operation's Leopard transform has at most 16 lanes (it runs
// in registers and ignores the FFT tile).
bool mix_fft_in_registers(Codec &c, int op);

// Planner (tuner.cu): overwrite plans[i] with the measured table's plan
// (RSGPU_PLANNER_TABLE and _MODEL) or, for classes the table has not
// measured, the cost model's best predicted plan (RSGPU_PLANNER_MODEL).
// Plans the planner has nothing for keep their incoming (default) value.
int mix_plan_batch(const rsgpu_mix_op *ops, size_t n, int planner, std::vector<rsgpu_plan> &plans);

}  // namespace rsgpu
