// batch.hpp -- mixed batches (batch.cu) and the plan selector (tuner.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <vector>

#include "rsgpu.h"

namespace rsgpu {

class Codec;
struct MixBatch;
struct MixDeleter {
  void operator()(MixBatch *b) const;
};
using MixPtr = std::unique_ptr<MixBatch, MixDeleter>;

// Prepare a mixed batch; `forced` (optional) gives every op's plan.
int mix_build(const rsgpu_mix_op *ops, size_t n_ops, const rsgpu_plan *forced, const rsgpu_mix_options &opt,
              MixPtr &out);
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
