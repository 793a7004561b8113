/*
 * rs_oracle.h -- CPU restatement of the rustfs-erasure-codec 9.1.0 hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against.  Only the test suite, the smoke check and the benchmark's
 * CPU-baseline leg may load it; the product library never links it and has no
 * CPU fallback.
 *
 * Every function follows a reference file cited at its definition (paths are
 * relative to the reference crate root).  Error codes are the reference
 * `Error` discriminant + 1 (src/errors.rs:3-21); 0 means success.
 */
#ifndef RS_ORACLE_H
#define RS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_OK = 0,
  ORC_TOO_FEW_SHARDS = 1,
  ORC_TOO_MANY_SHARDS = 2,
  ORC_TOO_FEW_DATA_SHARDS = 3,
  ORC_TOO_MANY_DATA_SHARDS = 4,
  ORC_TOO_FEW_PARITY_SHARDS = 5,
  ORC_TOO_MANY_PARITY_SHARDS = 6,
  ORC_TOO_FEW_BUFFER_SHARDS = 7,
  ORC_TOO_MANY_BUFFER_SHARDS = 8,
  ORC_INCORRECT_SHARD_SIZE = 9,
  ORC_TOO_FEW_SHARDS_PRESENT = 10,
  ORC_EMPTY_SHARD = 11,
  ORC_INVALID_SHARD_FLAGS = 12,
  ORC_INVALID_INDEX = 13,
  ORC_INVALID_CUSTOM_MATRIX = 14,
  ORC_UNSUPPORTED_CODEC_FAMILY = 15,
  ORC_UNSUPPORTED_LEOPARD_PROTOTYPE = 16,
};

/* ---- GF(2^8), poly 0x11d (build.rs:10-65, src/galois_8/mod.rs:139-183) ---- */
void orc_gf8_tables(uint8_t *log_table /*256*/, uint8_t *exp_table /*510*/);
uint8_t orc_gf8_mul(uint8_t a, uint8_t b);
uint8_t orc_gf8_div(uint8_t a, uint8_t b);
uint8_t orc_gf8_exp(uint8_t a, size_t n);
void orc_gf8_mul_slice(uint8_t c, const uint8_t *in, uint8_t *out, size_t len);
void orc_gf8_mul_slice_xor(uint8_t c, const uint8_t *in, uint8_t *out, size_t len);

/* ---- classic matrices (src/core/codec.rs:67-230, src/matrix.rs) ----
 * mode: 0 Vandermonde, 1 Cauchy, 2 JerasureLike, 3 Custom.
 * out: (k+m)*k row-major.  custom: m*k parity rows (mode 3 only). */
int orc_build_matrix(size_t k, size_t m, int mode, int fast_one_parity,
                     const uint8_t *custom, uint8_t *out);
/* Gauss-Jordan inverse of an n*n matrix; 0 or ORC_INVALID_CUSTOM_MATRIX. */
int orc_gf8_invert(size_t n, const uint8_t *in, uint8_t *out);

/* ---- classic codec over an explicit (k+m)*k matrix ---- */
void orc_classic_encode(size_t k, size_t m, const uint8_t *matrix,
                        const uint8_t *const *data, uint8_t *const *parity,
                        size_t len);
/* goal: 0 All, 1 Data, 2 Required (required has n_required entries, k or k+m).
 * present: k+m flags.  Missing targets are written in place. */
int orc_classic_reconstruct(size_t k, size_t m, const uint8_t *matrix,
                            uint8_t *const *shards, const uint8_t *present,
                            size_t len, int goal, const uint8_t *required,
                            size_t n_required);
/* Composed recovery rows used by the product path, exposed so tests can check
 * the row algebra directly: rows (n_out*k) over the first k present shards. */
int orc_classic_recovery_rows(size_t k, size_t m, const uint8_t *matrix,
                              const uint8_t *present, int goal,
                              const uint8_t *required, size_t n_required,
                              size_t *survivors /*k*/, size_t *targets,
                              size_t *n_targets, uint8_t *rows);
int orc_classic_verify(size_t k, size_t m, const uint8_t *matrix,
                       const uint8_t *const *shards, size_t len);
/* Progressive recovery (src/galois_8/policy.rs:543-700): NULL entries of dst /
 * input are None; expect == NULL selects merge mode. */
int orc_classic_decode_idx(size_t k, size_t m, const uint8_t *matrix, uint8_t *const *dst,
                           const size_t *dst_lens, size_t n_dst, const uint8_t *expect,
                           size_t n_expect, const uint8_t *const *input,
                           const size_t *input_lens, size_t n_input);

/* ---- Leopard GF(2^8) (src/core/leopard_gf8/) ---- */
void orc_lgf8_tables(uint8_t *log_lut, uint8_t *exp_lut, uint8_t *fft_skew /*255*/,
                     uint8_t *log_walsh);
uint8_t orc_lgf8_mul_log(uint8_t a, uint8_t log_b);
int orc_lgf8_encode(size_t k, size_t m, const uint8_t *const *data,
                    uint8_t *const *parity, size_t len);
int orc_lgf8_reconstruct(size_t k, size_t m, uint8_t *const *shards,
                         const uint8_t *present, const uint8_t *want, size_t len);
void orc_lgf8_error_locators(size_t k, size_t m, const uint8_t *present,
                             uint8_t *err_locs /*256*/);

/* ---- Leopard GF(2^16) (src/core/leopard_gf16/) ---- */
void orc_lgf16_tables(uint16_t *log_lut, uint16_t *exp_lut /*131072*/,
                      uint16_t *fft_skew /*65535*/, uint16_t *log_walsh);
uint16_t orc_lgf16_mul_log(uint16_t a, uint16_t log_b);
int orc_lgf16_encode(size_t k, size_t m, const uint8_t *const *data,
                     uint8_t *const *parity, size_t len);
int orc_lgf16_reconstruct(size_t k, size_t m, uint8_t *const *shards,
                          const uint8_t *present, const uint8_t *want, size_t len);
void orc_lgf16_error_locators(size_t k, size_t m, const uint8_t *present,
                              uint16_t *err_locs /*65536*/);

/* ---- classic GF(2^16) tower field (src/galois_16.rs) ---- */
void orc_gf16t_mul(const uint8_t *a, const uint8_t *b, uint8_t *out);
int orc_gf16t_build_matrix(size_t k, size_t m, uint8_t *out /*(k+m)*k*2*/);
void orc_gf16t_encode(size_t k, size_t m, const uint8_t *matrix,
                      const uint8_t *const *data, uint8_t *const *parity,
                      size_t len_elems);
int orc_gf16t_reconstruct(size_t k, size_t m, const uint8_t *matrix,
                          uint8_t *const *shards, const uint8_t *present,
                          size_t len_elems, int data_only);

/* ---- timed CPU baseline: threaded split-nibble classic encode ---- */
int orc_fast_encode_batch(size_t k, size_t m, const uint8_t *matrix,
                          uint8_t *const *shard_ptrs /* n_stripes*(k+m) */,
                          size_t n_stripes, size_t len, int threads);
const char *orc_fast_kernel_name(void);
/* Kernel choice of orc_fast_encode_batch: -1 = the host's widest GFNI (the
 * reference's selection order), 2 / 1 = GFNI at 64 / 32 bytes, 0 = nibble
 * tables; the best kernel the host supports is reported by
 * orc_fast_best_kernel. */
void orc_fast_force_kernel(int kernel);
int orc_fast_best_kernel(void);

#ifdef __cplusplus
}
#endif
#endif
