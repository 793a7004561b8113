// leopard.hpp -- family resolution plus the Leopard FFT and tower-field
// classic codecs (device pointers; validation already done by the caller).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <memory>

namespace rsgpu {

class Codec;

// A prepared Leopard (or tower-field) batch: device-resident job tables whose
// launch allocates and synchronizes nothing.
struct LeoLaunch;
int prepare_other(Codec &c, int op, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                  int goal, uint32_t *flags, std::shared_ptr<LeoLaunch> &out);
int leo_launch(const LeoLaunch &l, cudaStream_t s);
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

int tower_encode(Codec &c, size_t n_stripes, uint8_t *const *shards, size_t len, cudaStream_t s);
int tower_verify(Codec &c, size_t n_stripes, const uint8_t *const *shards, size_t len, uint8_t *ok,
                 cudaStream_t s);
int tower_reconstruct(Codec &c, size_t n_stripes, uint8_t *const *shards, const uint8_t *present, size_t len,
                      int goal, const uint8_t *required, size_t n_required, cudaStream_t s);

}  // namespace rsgpu
