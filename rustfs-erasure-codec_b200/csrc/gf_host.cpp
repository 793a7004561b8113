// gf_host.cpp -- construction-time field arithmetic (see gf_host.hpp).
#include "gf_host.hpp"

#include <cstring>

#include "common.hpp"
#include "rsgpu.h"

namespace rsgpu {

Gf8::Gf8() {
  // Repeated doubling modulo x^8 + x^4 + x^3 + x^2 + 1 enumerates the
  // multiplicative group in generator order (reference build.rs:10-25).
  std::memset(log, 0, sizeof(log));
  unsigned v = 1;
  for (unsigned e = 0; e < 255; ++e) {
    log[v] = static_cast<uint8_t>(e);
    exp[e] = exp[e + 255] = static_cast<uint8_t>(v);
    v <<= 1;
    if (v & 0x100) v ^= 0x11d;
  }
  for (unsigned a = 0; a < 256; ++a)
    for (unsigned b = 0; b < 256; ++b)
      mul[a][b] = (a && b) ? exp[log[a] + log[b]] : 0;
}

uint8_t Gf8::div(uint8_t a, uint8_t b) const {
  // Zero for a zero operand (src/galois_8/mod.rs:155-166).
  if (!a || !b) return 0;
  int e = int(log[a]) - int(log[b]);
  return exp[e < 0 ? e + 255 : e];
}

uint8_t Gf8::pow(uint8_t a, size_t n) const {
  // 0^0 = 1; exponents reduce modulo the group order (src/galois_8/mod.rs:168-183).
  if (n == 0) return 1;
  if (a == 0) return 0;
  return exp[(size_t(log[a]) * (n % 255)) % 255];
}

const Gf8 &gf8() {
  static const Gf8 f;
  return f;
}

// ---------------------------------------------------------------- tower field
T16 t16_mul(T16 a, T16 b) {
  // (ax X + ac)(bx X + bc) with X^2 = 2X + 128.
  const Gf8 &f = gf8();
  uint8_t hi = f.mul[a.x][b.x];
  uint8_t mid = f.mul[a.c][b.x] ^ f.mul[a.x][b.c];
  uint8_t lo = f.mul[a.c][b.c];
  return T16{uint8_t(mid ^ f.mul[2][hi]), uint8_t(lo ^ f.mul[128][hi])};
}

T16 t16_inv(T16 a) {
  // Conjugate over the norm; the inverse of zero is zero (src/galois_16.rs:659-680).
  const Gf8 &f = gf8();
  if (a.x == 0) return T16{0, uint8_t(a.c ? f.inv(a.c) : 0)};
  uint8_t conj = a.c ^ f.mul[2][a.x];
  uint8_t norm = f.mul[a.c][conj] ^ f.mul[128][f.mul[a.x][a.x]];
  uint8_t ni = f.inv(norm);
  return T16{f.mul[a.x][ni], f.mul[conj][ni]};
}

T16 t16_pow(T16 a, size_t n) {
  if (n == 0) return T16{0, 1};
  if (t16_zero(a)) return T16{0, 0};
  n %= 65535;
  T16 r{0, 1}, base = a;
  while (n) {
    if (n & 1) r = t16_mul(r, base);
    base = t16_mul(base, base);
    n >>= 1;
  }
  return r;
}

// ---------------------------------------------------------------- matrices
namespace {

// Generic Gauss-Jordan on an augmented [A | I] system of n rows.  Pivoting
// takes the first nonzero entry at or below the diagonal; the inverse is
// unique, so only the singularity verdict depends on the elimination order.
template <class E, class Ops>
bool invert_generic(size_t n, const E *in, E *out, const Ops &ops) {
  const size_t w = 2 * n;
  std::vector<E> a(n * w, ops.zero());
  for (size_t r = 0; r < n; ++r) {
    for (size_t c = 0; c < n; ++c) a[r * w + c] = in[r * n + c];
    a[r * w + n + r] = ops.one();
  }
  for (size_t col = 0; col < n; ++col) {
    size_t p = col;
    while (p < n && ops.is_zero(a[p * w + col])) ++p;
    if (p == n) return false;
    if (p != col)
      for (size_t c = 0; c < w; ++c) std::swap(a[p * w + c], a[col * w + c]);
    E s = ops.inv(a[col * w + col]);
    for (size_t c = 0; c < w; ++c) a[col * w + c] = ops.mul(s, a[col * w + c]);
    for (size_t r = 0; r < n; ++r) {
      if (r == col) continue;
      E f = a[r * w + col];
      if (ops.is_zero(f)) continue;
      for (size_t c = 0; c < w; ++c) a[r * w + c] = ops.add(a[r * w + c], ops.mul(f, a[col * w + c]));
    }
  }
  for (size_t r = 0; r < n; ++r)
    for (size_t c = 0; c < n; ++c) out[r * n + c] = a[r * w + n + c];
  return true;
}

struct Ops8 {
  uint8_t zero() const { return 0; }
  uint8_t one() const { return 1; }
  bool is_zero(uint8_t a) const { return a == 0; }
  uint8_t inv(uint8_t a) const { return gf8().inv(a); }
  uint8_t mul(uint8_t a, uint8_t b) const { return gf8().mul[a][b]; }
  uint8_t add(uint8_t a, uint8_t b) const { return a ^ b; }
};
struct Ops16 {
  T16 zero() const { return T16{0, 0}; }
  T16 one() const { return T16{0, 1}; }
  bool is_zero(T16 a) const { return t16_zero(a); }
  T16 inv(T16 a) const { return t16_inv(a); }
  T16 mul(T16 a, T16 b) const { return t16_mul(a, b); }
  T16 add(T16 a, T16 b) const { return T16{uint8_t(a.x ^ b.x), uint8_t(a.c ^ b.c)}; }
};

}  // namespace

bool gf8_invert(size_t n, const uint8_t *in, uint8_t *out) {
  return invert_generic(n, in, out, Ops8{});
}

bool t16_invert(size_t n, const T16 *in, T16 *out) {
  return invert_generic(n, in, out, Ops16{});
}

int build_encoding_matrix(size_t k, size_t m, int mode, bool fast_one_parity,
                          const uint8_t *custom_rows, Mat8 &out) {
  const Gf8 &f = gf8();
  const size_t total = k + m;
  out.assign(total * k, 0);
  auto at = [&](size_t r, size_t c) -> uint8_t & { return out[r * k + c]; };

  if (mode == RSGPU_MATRIX_CUSTOM) {
    // Identity data rows over the caller's parity rows (src/core/codec.rs:196-226);
    // single-parity fast mode requires an all-ones row (:594-603).
    for (size_t r = 0; r < k; ++r) at(r, r) = 1;
    std::memcpy(&out[k * k], custom_rows, m * k);
    if (fast_one_parity && m == 1)
      for (size_t c = 0; c < k; ++c)
        if (at(k, c) != 1) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
    return RSGPU_OK;
  }
  if (fast_one_parity && m == 1) {
    // Single-parity XOR format (src/core/codec.rs:236-247).
    for (size_t c = 0; c < k; ++c) at(c, c) = at(k, c) = 1;
    return RSGPU_OK;
  }
  if (mode == RSGPU_MATRIX_CAUCHY) {
    // Identity over 1 / (r + c) (src/core/codec.rs:91-110).
    for (size_t r = 0; r < k; ++r) at(r, r) = 1;
    for (size_t r = k; r < total; ++r)
      for (size_t c = 0; c < k; ++c) {
        uint8_t d = uint8_t(r) ^ uint8_t(c);
        if (!d) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
        at(r, c) = f.inv(d);
      }
    return RSGPU_OK;
  }

  // Vandermonde rows r^c with r taken as a field element (src/matrix.rs:446-459).
  Mat8 v(total * k);
  for (size_t r = 0; r < total; ++r)
    for (size_t c = 0; c < k; ++c) v[r * k + c] = f.pow(uint8_t(r), c);

  if (mode == RSGPU_MATRIX_VANDERMONDE) {
    // V * inverse(top k rows of V) (src/core/codec.rs:67-89).
    Mat8 inv(k * k);
    if (!gf8_invert(k, v.data(), inv.data())) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
    for (size_t r = 0; r < total; ++r)
      for (size_t i = 0; i < k; ++i) {
        uint8_t co = v[r * k + i];
        if (!co)
          continue;
        for (size_t c = 0; c < k; ++c) at(r, c) ^= f.mul[co][inv[i * k + c]];
      }
    return RSGPU_OK;
  }

  if (mode == RSGPU_MATRIX_JERASURE_LIKE) {
    // Column reduction of a modified Vandermonde matrix followed by row and
    // column normalisation of the parity block (src/core/codec.rs:112-194).
    out = v;
    at(0, 0) = 1;
    for (size_t c = 1; c < k; ++c) at(0, c) = 0;
    for (size_t c = 0; c + 1 < k; ++c) at(total - 1, c) = 0;
    at(total - 1, k - 1) = 1;
    for (size_t i = 0; i < k; ++i) {
      size_t r = i;
      while (r < total && at(r, i) == 0) ++r;
      if (r == total) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
      if (r != i)
        for (size_t c = 0; c < k; ++c) std::swap(at(r, c), at(i, c));
      uint8_t dgl = at(i, i);
      if (!dgl) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
      if (dgl != 1) {
        uint8_t s = f.inv(dgl);
        for (size_t row = 0; row < total; ++row) at(row, i) = f.mul[at(row, i)][s];
      }
      for (size_t j = 0; j < k; ++j) {
        uint8_t val = at(i, j);
        if (j == i || !val) continue;
        for (size_t row = 0; row < total; ++row) at(row, j) ^= f.mul[val][at(row, i)];
      }
    }
    for (size_t j = 0; j < k; ++j) {
      uint8_t val = at(k, j);
      if (!val) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
      if (val != 1) {
        uint8_t s = f.inv(val);
        for (size_t row = k; row < total; ++row) at(row, j) = f.mul[at(row, j)][s];
      }
    }
    for (size_t row = k + 1; row < total; ++row) {
      uint8_t val = at(row, 0);
      if (!val) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
      if (val != 1) {
        uint8_t s = f.inv(val);
        for (size_t c = 0; c < k; ++c) at(row, c) = f.mul[at(row, c)][s];
      }
    }
    return RSGPU_OK;
  }
  return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
}

int build_tower_matrix(size_t k, size_t m, std::vector<T16> &out) {
  const size_t total = k + m;
  std::vector<T16> v(total * k), inv(k * k);
  for (size_t r = 0; r < total; ++r) {
    T16 a{uint8_t(r >> 8), uint8_t(r)};  // nth(r) (src/galois_16.rs:63-65)
    for (size_t c = 0; c < k; ++c) v[r * k + c] = t16_pow(a, c);
  }
  if (!t16_invert(k, v.data(), inv.data())) return RSGPU_ERR_INVALID_CUSTOM_MATRIX;
  out.assign(total * k, T16{0, 0});
  for (size_t r = 0; r < total; ++r)
    for (size_t i = 0; i < k; ++i) {
      T16 co = v[r * k + i];
      if (t16_zero(co)) continue;
      for (size_t c = 0; c < k; ++c) {
        T16 p = t16_mul(co, inv[i * k + c]);
        out[r * k + c].x ^= p.x;
        out[r * k + c].c ^= p.c;
      }
    }
  return RSGPU_OK;
}

void pack_tables(const uint8_t *rows, size_t n_out, size_t n_in, uint32_t *out) {
  pack_tables_with(gf8().mul, rows, n_out, n_in, out);
}

void pack_tables_with(const uint8_t (*mul)[256], const uint8_t *rows, size_t n_out, size_t n_in, uint32_t *out) {
  const size_t groups = (n_out + 3) / 4;
  for (size_t g = 0; g < groups; ++g)
    for (size_t j = 0; j < n_in; ++j) {
      uint32_t *t = out + (g * n_in + j) * kTableWords;
      for (unsigned i = 0; i < unsigned(kTableWords); ++i) t[i] = 0;
      for (unsigned r = 0; r < 4; ++r) {
        const size_t o = g * 4 + r;
        if (o >= n_out) break;
        const uint8_t c = rows[o * n_in + j];
        for (unsigned n = 0; n < 16; ++n) {
          t[n] |= uint32_t(mul[c][n]) << (8 * r);
          t[16 + n] |= uint32_t(mul[c][n << 4]) << (8 * r);
        }
        for (unsigned i = 0; i < 32; ++i) t[32 + i] |= uint32_t(mul[c][i]) << (8 * r);
        for (unsigned h = 0; h < 8; ++h) t[64 + 2 * r + (h >> 2)] |= uint32_t(mul[c][h << 5]) << (8 * (h & 3));
      }
    }
}

}  // namespace rsgpu
