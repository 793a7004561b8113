// model.hpp -- the planner's learned cost model (model.cu).
#pragma once

#include <cstddef>
#include <cstdint>

#include "rsgpu.h"

namespace rsgpu {

size_t model_param_count();
bool model_ready();
int model_get(float *out, size_t n);
int model_set(const float *in, size_t n);
// Forward pass on the GPU for n feature rows (rows seen before under the
// same weights come from a memo when `memoize`); *version (optional) gets the
// weight set's version, which model_set advances.
int model_predict(const float *features, size_t n, float *out, bool memoize = true, uint64_t *version = nullptr);
uint64_t model_version();
int model_gradients(const float *params, const float *features, const float *targets, const uint8_t *mask, size_t n,
                    float *loss, float *grads);
int model_train(const float *features, const float *targets, const uint8_t *mask, size_t n,
                const rsgpu_train_options &o, float *final_loss);

}  // namespace rsgpu
