// gf_host.hpp -- host-side field arithmetic used to set up codecs.
//
// GF(2^8) with polynomial 0x11d and generator 2 (reference build.rs:10-65),
// and the GF((2^8)^2) tower field with X^2 = 2X + 128 (src/galois_16.rs:9-11).
// Only construction-time work runs here (encoding matrices and table
// packing); all per-byte arithmetic runs on the GPU.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace rsgpu {

struct Gf8 {
  uint8_t log[256];
  uint8_t exp[510];
  uint8_t mul[256][256];
  Gf8();
  uint8_t div(uint8_t a, uint8_t b) const;
  uint8_t pow(uint8_t a, size_t n) const;
  uint8_t inv(uint8_t a) const { return div(1, a); }
};
const Gf8 &gf8();

// Tower element x*X + c stored as bytes {x, c}.
struct T16 {
  uint8_t x, c;
};
T16 t16_mul(T16 a, T16 b);
T16 t16_inv(T16 a);
T16 t16_pow(T16 a, size_t n);
inline bool t16_zero(T16 a) { return a.x == 0 && a.c == 0; }

// Dense matrices over GF(2^8), row-major.
using Mat8 = std::vector<uint8_t>;
// Gauss-Jordan inverse; false when singular.
bool gf8_invert(size_t n, const uint8_t *in, uint8_t *out);
// Classic encoding matrix (k+m rows, k columns).  mode: RSGPU_MATRIX_*.
// Returns 0 or an RSGPU_ERR_* code.
int build_encoding_matrix(size_t k, size_t m, int mode, bool fast_one_parity,
                          const uint8_t *custom_rows, Mat8 &out);

// Tower-field matrices: 2 bytes per entry.
bool t16_invert(size_t n, const T16 *in, T16 *out);
int build_tower_matrix(size_t k, size_t m, std::vector<T16> &out);

// Nibble tables for the matrix-apply kernel; rows is n_out x n_in.
void pack_tables(const uint8_t *rows, size_t n_out, size_t n_in, uint32_t *out);
// The same layout for any GF(2)-linear byte field: mul[c][x] = c * x.
void pack_tables_with(const uint8_t (*mul)[256], const uint8_t *rows, size_t n_out, size_t n_in, uint32_t *out);

}  // namespace rsgpu
