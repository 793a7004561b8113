// pending.cpp -- families whose device path is not wired up yet report
// UnsupportedCodecFamily instead of computing anything on the CPU.
#include "codec.hpp"
#include "leopard.hpp"

namespace rsgpu {
struct LeopardState {};
int Codec::init_tower() { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int Codec::init_leopard() { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int leopard_encode(Codec &, size_t, uint8_t *const *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int leopard_verify(Codec &, size_t, const uint8_t *const *, size_t, uint8_t *, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int leopard_reconstruct(Codec &, size_t, uint8_t *const *, const uint8_t *, size_t, int, const uint8_t *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int tower_encode(Codec &, size_t, uint8_t *const *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int tower_verify(Codec &, size_t, const uint8_t *const *, size_t, uint8_t *, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int tower_reconstruct(Codec &, size_t, uint8_t *const *, const uint8_t *, size_t, int, const uint8_t *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
}  // namespace rsgpu
