// pending.cpp -- families whose device path is not wired up yet report
// UnsupportedCodecFamily instead of computing anything on the CPU.
#include "codec.hpp"
#include "leopard.hpp"

namespace rsgpu {
struct LeopardState {};
struct LeoLaunch {};
int prepare_other(Codec &, int, size_t, uint8_t *const *, const uint8_t *, size_t, int, uint32_t *, std::shared_ptr<LeoLaunch> &) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int leo_launch(const LeoLaunch &, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
uint32_t leo_kernel_count(const LeoLaunch &) { return 0; }
int Codec::init_tower() { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int Codec::init_leopard() { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int leopard_encode(Codec &, size_t, uint8_t *const *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int leopard_verify(Codec &, size_t, const uint8_t *const *, size_t, uint8_t *, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int leopard_reconstruct(Codec &, size_t, uint8_t *const *, const uint8_t *, size_t, int, const uint8_t *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int tower_encode(Codec &, size_t, uint8_t *const *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int tower_verify(Codec &, size_t, const uint8_t *const *, size_t, uint8_t *, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
int tower_reconstruct(Codec &, size_t, uint8_t *const *, const uint8_t *, size_t, int, const uint8_t *, size_t, cudaStream_t) { return RSGPU_ERR_UNSUPPORTED_CODEC_FAMILY; }
}  // namespace rsgpu
