/*
 * gf16_tower.c -- oracle restatement of the classic GF((2^8)^2) tower field
 * codec (src/galois_16.rs) of rustfs-erasure-codec 9.1.0.  TEST
 * INFRASTRUCTURE ONLY (see rs_oracle.h).
 *
 * An element is the byte pair [x, c] meaning x*X + c, with X^2 = 2X + 128
 * (EXT_POLY = [1, 2, 128], src/galois_16.rs:9-11).  The codec is the generic
 * classic codec of src/core/ instantiated with this field.
 */
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

typedef struct {
  uint8_t x, c;
} t16;

static t16 tmul(t16 a, t16 b) {
  /* src/galois_16.rs:730-746 (FOIL) and :684-694 (reduce_from). */
  uint8_t o0 = orc_gf8_mul(a.x, b.x);
  uint8_t o1 = orc_gf8_mul(a.c, b.x) ^ orc_gf8_mul(a.x, b.c);
  uint8_t o2 = orc_gf8_mul(a.c, b.c);
  if (o0 != 0) {
    o1 ^= orc_gf8_mul(2, o0);
    o2 ^= orc_gf8_mul(128, o0);
  }
  t16 r = {o1, o2};
  return r;
}

/* src/galois_16.rs:659-680 */
static t16 tinv(t16 a) {
  t16 r = {0, 0};
  if (a.x == 0) {
    if (a.c != 0) r.c = orc_gf8_div(1, a.c);
    return r;
  }
  uint8_t conj = a.c ^ orc_gf8_mul(2, a.x);
  uint8_t norm = orc_gf8_mul(a.c, conj) ^ orc_gf8_mul(128, orc_gf8_mul(a.x, a.x));
  uint8_t ni = orc_gf8_div(1, norm);
  r.x = orc_gf8_mul(a.x, ni);
  r.c = orc_gf8_mul(conj, ni);
  return r;
}

/* src/galois_16.rs:630-655 */
static t16 texp(t16 a, size_t n) {
  t16 one = {0, 1}, zero = {0, 0};
  if (n == 0) return one;
  if (a.x == 0 && a.c == 0) return zero;
  n %= 65535;
  if (n == 0) return one;
  size_t top = 1;
  while ((top << 1) <= n) top <<= 1;
  t16 p = a;
  for (size_t bit = top >> 1; bit; bit >>= 1) {
    p = tmul(p, p);
    if (n & bit) p = tmul(p, a);
  }
  return p;
}

void orc_gf16t_mul(const uint8_t *a, const uint8_t *b, uint8_t *out) {
  t16 x = {a[0], a[1]}, y = {b[0], b[1]};
  t16 r = tmul(x, y);
  out[0] = r.x;
  out[1] = r.c;
}

static int tinvert(size_t n, const t16 *in, t16 *out) {
  size_t cols = 2 * n;
  t16 *w = (t16 *)calloc(n * cols, sizeof(t16));
  for (size_t r = 0; r < n; r++) {
    memcpy(w + r * cols, in + r * n, n * sizeof(t16));
    w[r * cols + n + r].c = 1;
  }
  int rc = ORC_OK;
#define W(r, c) w[(r) * cols + (c)]
#define ISZ(e) ((e).x == 0 && (e).c == 0)
  for (size_t r = 0; r < n && rc == ORC_OK; r++) {
    if (ISZ(W(r, r)))
      for (size_t rb = r + 1; rb < n; rb++)
        if (!ISZ(W(rb, r))) {
          for (size_t c = 0; c < cols; c++) {
            t16 t = W(r, c);
            W(r, c) = W(rb, c);
            W(rb, c) = t;
          }
          break;
        }
    if (ISZ(W(r, r))) {
      rc = ORC_INVALID_CUSTOM_MATRIX;
      break;
    }
    t16 s = tinv(W(r, r));
    for (size_t c = 0; c < cols; c++) W(r, c) = tmul(s, W(r, c));
    for (size_t rb = r + 1; rb < n; rb++) {
      t16 f = W(rb, r);
      if (ISZ(f)) continue;
      for (size_t c = 0; c < cols; c++) {
        t16 p = tmul(f, W(r, c));
        W(rb, c).x ^= p.x;
        W(rb, c).c ^= p.c;
      }
    }
  }
  for (size_t d = 0; d < n && rc == ORC_OK; d++)
    for (size_t ra = 0; ra < d; ra++) {
      t16 f = W(ra, d);
      if (ISZ(f)) continue;
      for (size_t c = 0; c < cols; c++) {
        t16 p = tmul(f, W(d, c));
        W(ra, c).x ^= p.x;
        W(ra, c).c ^= p.c;
      }
    }
  if (rc == ORC_OK)
    for (size_t r = 0; r < n; r++) memcpy(out + r * n, w + r * cols + n, n * sizeof(t16));
#undef W
#undef ISZ
  free(w);
  return rc;
}

/* src/core/codec.rs:67-89 with nth(n) = [(n >> 8), n] (galois_16.rs:63-65). */
int orc_gf16t_build_matrix(size_t k, size_t m, uint8_t *out) {
  size_t total = k + m;
  t16 *v = (t16 *)calloc(total * k + 1, sizeof(t16));
  t16 *inv = (t16 *)malloc(k * k * sizeof(t16));
  for (size_t r = 0; r < total; r++) {
    t16 a = {(uint8_t)(r >> 8), (uint8_t)r};
    for (size_t c = 0; c < k; c++) v[r * k + c] = texp(a, c);
  }
  int rc = tinvert(k, v, inv);
  if (rc == ORC_OK)
    for (size_t r = 0; r < total; r++)
      for (size_t c = 0; c < k; c++) {
        t16 acc = {0, 0};
        for (size_t i = 0; i < k; i++) {
          t16 p = tmul(v[r * k + i], inv[i * k + c]);
          acc.x ^= p.x;
          acc.c ^= p.c;
        }
        out[(r * k + c) * 2] = acc.x;
        out[(r * k + c) * 2 + 1] = acc.c;
      }
  free(v);
  free(inv);
  return rc;
}

static void apply_row(const uint8_t *row, size_t n_in, const uint8_t *const *in, uint8_t *out,
                      size_t len_elems) {
  memset(out, 0, len_elems * 2);
  for (size_t j = 0; j < n_in; j++) {
    t16 co = {row[2 * j], row[2 * j + 1]};
    for (size_t e = 0; e < len_elems; e++) {
      t16 a = {in[j][2 * e], in[j][2 * e + 1]};
      t16 p = tmul(co, a);
      out[2 * e] ^= p.x;
      out[2 * e + 1] ^= p.c;
    }
  }
}

void orc_gf16t_encode(size_t k, size_t m, const uint8_t *matrix, const uint8_t *const *data,
                      uint8_t *const *parity, size_t len_elems) {
  for (size_t r = 0; r < m; r++) apply_row(matrix + (k + r) * k * 2, k, data, parity[r], len_elems);
}

/* Two-stage classic recovery (src/core/reconstruct.rs:318-416) over the tower
 * field: inverse rows on the first k present shards, then encoding rows on
 * the completed data. */
int orc_gf16t_reconstruct(size_t k, size_t m, const uint8_t *matrix, uint8_t *const *shards,
                          const uint8_t *present, size_t len_elems, int data_only) {
  size_t total = k + m, ns = 0, np = 0;
  size_t surv[512];
  int missing_data = 0, missing_any = 0;
  for (size_t i = 0; i < total; i++) {
    if (present[i]) {
      np++;
      if (ns < k) surv[ns++] = i;
    } else {
      missing_any = 1;
      if (i < k) missing_data = 1;
    }
  }
  if (!missing_any) return ORC_OK;
  if (np < k) return ORC_TOO_FEW_SHARDS_PRESENT;
  if (missing_data) {
    t16 *sel = (t16 *)calloc(k * k + 1, sizeof(t16));
    t16 *dec = (t16 *)malloc(k * k * sizeof(t16));
    for (size_t r = 0; r < k; r++)
      for (size_t c = 0; c < k; c++) {
        sel[r * k + c].x = matrix[(surv[r] * k + c) * 2];
        sel[r * k + c].c = matrix[(surv[r] * k + c) * 2 + 1];
      }
    int rc = tinvert(k, sel, dec);
    if (rc != ORC_OK) {
      free(sel);
      free(dec);
      return rc;
    }
    const uint8_t **in = (const uint8_t **)malloc(k * sizeof(uint8_t *));
    for (size_t c = 0; c < k; c++) in[c] = shards[surv[c]];
    uint8_t *row = (uint8_t *)malloc(k * 2);
    uint8_t *tmp = (uint8_t *)malloc(len_elems * 2 * k + 2);
    for (size_t d = 0; d < k; d++) {
      if (present[d]) continue;
      for (size_t c = 0; c < k; c++) {
        row[2 * c] = dec[d * k + c].x;
        row[2 * c + 1] = dec[d * k + c].c;
      }
      apply_row(row, k, in, tmp + d * len_elems * 2, len_elems);
    }
    for (size_t d = 0; d < k; d++)
      if (!present[d]) memcpy(shards[d], tmp + d * len_elems * 2, len_elems * 2);
    free(tmp);
    free(row);
    free(in);
    free(sel);
    free(dec);
  }
  if (!data_only)
    for (size_t p = k; p < total; p++)
      if (!present[p])
        apply_row(matrix + p * k * 2, k, (const uint8_t *const *)shards, shards[p], len_elems);
  return ORC_OK;
}
