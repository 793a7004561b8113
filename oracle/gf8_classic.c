/*
 * gf8_classic.c -- oracle restatement of the classic GF(2^8) Reed-Solomon
 * codec of rustfs-erasure-codec 9.1.0.  TEST INFRASTRUCTURE ONLY (see
 * rs_oracle.h): the checker for the CUDA path, never the thing measured.
 */
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

static uint8_t LOG8[256];
static uint8_t EXP8[510];
static uint8_t MUL8[256][256];
static int gf8_ready;

/* build.rs:10-65: log table by repeated doubling modulo x^8+x^4+x^3+x^2+1
 * (GENERATING_POLYNOMIAL 29 after dropping bit 8), a 510-entry exp table with
 * its wrap-around copy, and the full product table. */
static void gf8_init(void) {
  if (gf8_ready) return;
  unsigned b = 1;
  for (unsigned lg = 0; lg < 255; lg++) {
    LOG8[b] = (uint8_t)lg;
    b <<= 1;
    if (b >= 256) b = (b - 256) ^ 29u;
  }
  for (unsigned i = 1; i < 256; i++) {
    unsigned l = LOG8[i];
    EXP8[l] = (uint8_t)i;
    EXP8[l + 255] = (uint8_t)i;
  }
  for (unsigned a = 0; a < 256; a++)
    for (unsigned c = 0; c < 256; c++)
      MUL8[a][c] = (a == 0 || c == 0) ? 0 : EXP8[LOG8[a] + LOG8[c]];
  gf8_ready = 1;
}

void orc_gf8_tables(uint8_t *log_table, uint8_t *exp_table) {
  gf8_init();
  memcpy(log_table, LOG8, 256);
  memcpy(exp_table, EXP8, 510);
}

/* src/galois_8/mod.rs:139-141 */
uint8_t orc_gf8_mul(uint8_t a, uint8_t b) {
  gf8_init();
  return MUL8[a][b];
}

/* src/galois_8/mod.rs:155-166: zero when either operand is zero. */
uint8_t orc_gf8_div(uint8_t a, uint8_t b) {
  gf8_init();
  if (a == 0 || b == 0) return 0;
  int l = (int)LOG8[a] - (int)LOG8[b];
  if (l < 0) l += 255;
  return EXP8[l];
}

/* src/galois_8/mod.rs:168-183: 0^0 = 1, exponent reduced mod 255. */
uint8_t orc_gf8_exp(uint8_t a, size_t n) {
  gf8_init();
  if (n == 0) return 1;
  if (a == 0) return 0;
  size_t l = ((size_t)LOG8[a] * (n % 255)) % 255;
  return EXP8[l];
}

void orc_gf8_mul_slice(uint8_t c, const uint8_t *in, uint8_t *out, size_t len) {
  gf8_init();
  for (size_t i = 0; i < len; i++) out[i] = MUL8[c][in[i]];
}

void orc_gf8_mul_slice_xor(uint8_t c, const uint8_t *in, uint8_t *out, size_t len) {
  gf8_init();
  for (size_t i = 0; i < len; i++) out[i] ^= MUL8[c][in[i]];
}

/* ------------------------------------------------------------------------ */
/* Matrices (src/matrix.rs).  Row-major, rows*cols bytes.                    */

static void swap_rows(uint8_t *a, size_t cols, size_t r1, size_t r2) {
  if (r1 == r2) return;
  for (size_t i = 0; i < cols; i++) {
    uint8_t t = a[r1 * cols + i];
    a[r1 * cols + i] = a[r2 * cols + i];
    a[r2 * cols + i] = t;
  }
}

/* src/matrix.rs:373-422: forward elimination with "first nonzero row below"
 * pivoting, unit scaling, then back substitution in column order. */
static int gaussian_elim(uint8_t *a, size_t rows, size_t cols) {
  for (size_t r = 0; r < rows; r++) {
    if (a[r * cols + r] == 0) {
      for (size_t rb = r + 1; rb < rows; rb++) {
        if (a[rb * cols + r] != 0) {
          swap_rows(a, cols, r, rb);
          break;
        }
      }
    }
    if (a[r * cols + r] == 0) return -1; /* singular */
    if (a[r * cols + r] != 1) {
      uint8_t scale = orc_gf8_div(1, a[r * cols + r]);
      for (size_t c = 0; c < cols; c++) a[r * cols + c] = MUL8[scale][a[r * cols + c]];
    }
    for (size_t rb = r + 1; rb < rows; rb++) {
      uint8_t s = a[rb * cols + r];
      if (s != 0)
        for (size_t c = 0; c < cols; c++) a[rb * cols + c] ^= MUL8[s][a[r * cols + c]];
    }
  }
  for (size_t d = 0; d < rows; d++) {
    for (size_t ra = 0; ra < d; ra++) {
      uint8_t s = a[ra * cols + d];
      if (s != 0)
        for (size_t c = 0; c < cols; c++) a[ra * cols + c] ^= MUL8[s][a[d * cols + c]];
    }
  }
  return 0;
}

/* src/matrix.rs:424-444: invert via [A | I]. */
int orc_gf8_invert(size_t n, const uint8_t *in, uint8_t *out) {
  gf8_init();
  uint8_t *w = (uint8_t *)calloc(n * 2 * n, 1);
  for (size_t r = 0; r < n; r++) {
    memcpy(w + r * 2 * n, in + r * n, n);
    w[r * 2 * n + n + r] = 1;
  }
  int rc = gaussian_elim(w, n, 2 * n);
  if (rc == 0)
    for (size_t r = 0; r < n; r++) memcpy(out + r * n, w + r * 2 * n + n, n);
  free(w);
  return rc == 0 ? ORC_OK : ORC_INVALID_CUSTOM_MATRIX;
}

/* src/matrix.rs:446-459: entry (r, c) = exp(nth(r), c) with nth(r) = r as u8. */
static void vandermonde(uint8_t *v, size_t rows, size_t cols) {
  for (size_t r = 0; r < rows; r++)
    for (size_t c = 0; c < cols; c++) v[r * cols + c] = orc_gf8_exp((uint8_t)r, c);
}

/* src/matrix.rs:195-214 */
static void mat_mul(const uint8_t *a, size_t ar, size_t ac, const uint8_t *b, size_t bc,
                    uint8_t *out) {
  memset(out, 0, ar * bc);
  for (size_t r = 0; r < ar; r++)
    for (size_t i = 0; i < ac; i++) {
      uint8_t co = a[r * ac + i];
      if (co == 0) continue;
      for (size_t c = 0; c < bc; c++) out[r * bc + c] ^= MUL8[co][b[i * bc + c]];
    }
}

/* src/core/codec.rs:67-89: V * inv(V_top). */
static int build_vandermonde(size_t k, size_t total, uint8_t *out) {
  uint8_t *v = (uint8_t *)malloc(total * k);
  uint8_t *inv = (uint8_t *)malloc(k * k);
  vandermonde(v, total, k);
  int rc = orc_gf8_invert(k, v, inv);
  if (rc == ORC_OK) mat_mul(v, total, k, inv, k, out);
  free(v);
  free(inv);
  return rc;
}

/* src/core/codec.rs:91-110 */
static int build_cauchy(size_t k, size_t total, uint8_t *out) {
  memset(out, 0, total * k);
  for (size_t r = 0; r < total; r++) {
    if (r < k) {
      out[r * k + r] = 1;
      continue;
    }
    for (size_t c = 0; c < k; c++) {
      uint8_t den = (uint8_t)r ^ (uint8_t)c;
      if (den == 0) return ORC_INVALID_CUSTOM_MATRIX;
      out[r * k + c] = orc_gf8_div(1, den);
    }
  }
  return ORC_OK;
}

/* src/core/codec.rs:112-194.  The reference indexes one row past the end when
 * a pivot column is all zero below the diagonal (a panic); that case is
 * reported here as InvalidCustomMatrix. */
static int build_jerasure_like(size_t k, size_t total, uint8_t *vm) {
  vandermonde(vm, total, k);
#define VM(r, c) vm[(r) * k + (c)]
  VM(0, 0) = 1;
  for (size_t i = 1; i < k; i++) VM(0, i) = 0;
  for (size_t i = 0; i + 1 < k; i++) VM(total - 1, i) = 0;
  VM(total - 1, k - 1) = 1;
  for (size_t i = 0; i < k; i++) {
    size_t r = i;
    while (r < total && VM(r, i) == 0) r++;
    if (r == total) return ORC_INVALID_CUSTOM_MATRIX;
    if (r != i)
      swap_rows(vm, k, r, i);
    else if (VM(i, i) == 0)
      return ORC_INVALID_CUSTOM_MATRIX;
    uint8_t diag = VM(i, i);
    if (diag == 0) return ORC_INVALID_CUSTOM_MATRIX;
    uint8_t scale = diag != 1 ? orc_gf8_div(1, diag) : 1;
    if (scale != 1)
      for (size_t row = 0; row < total; row++) VM(row, i) = MUL8[VM(row, i)][scale];
    for (size_t j = 0; j < k; j++) {
      uint8_t value = VM(i, j);
      if (j != i && value != 0)
        for (size_t row = 0; row < total; row++) VM(row, j) ^= MUL8[value][VM(row, i)];
    }
  }
  for (size_t j = 0; j < k; j++) {
    uint8_t value = VM(k, j);
    if (value == 0) return ORC_INVALID_CUSTOM_MATRIX;
    if (value != 1) {
      uint8_t scale = orc_gf8_div(1, value);
      for (size_t row = k; row < total; row++) VM(row, j) = MUL8[VM(row, j)][scale];
    }
  }
  for (size_t row = k + 1; row < total; row++) {
    uint8_t value = VM(row, 0);
    if (value == 0) return ORC_INVALID_CUSTOM_MATRIX;
    if (value != 1) {
      uint8_t scale = orc_gf8_div(1, value);
      for (size_t col = 0; col < k; col++) VM(row, col) = MUL8[VM(row, col)][scale];
    }
  }
#undef VM
  return ORC_OK;
}

/* src/core/codec.rs:229-258 (build_matrix_with_options) and :196-226
 * (build_custom_matrix). */
int orc_build_matrix(size_t k, size_t m, int mode, int fast_one_parity,
                     const uint8_t *custom, uint8_t *out) {
  gf8_init();
  size_t total = k + m;
  if (mode == 3) {
    memset(out, 0, total * k);
    for (size_t r = 0; r < k; r++) out[r * k + r] = 1;
    for (size_t p = 0; p < m; p++) memcpy(out + (k + p) * k, custom + p * k, k);
    if (fast_one_parity && m == 1)
      for (size_t c = 0; c < k; c++)
        if (out[k * k + c] != 1) return ORC_INVALID_CUSTOM_MATRIX;
    return ORC_OK;
  }
  if (fast_one_parity && total == k + 1) {
    memset(out, 0, total * k);
    for (size_t c = 0; c < k; c++) {
      out[c * k + c] = 1;
      out[k * k + c] = 1;
    }
    return ORC_OK;
  }
  switch (mode) {
    case 0: return build_vandermonde(k, total, out);
    case 1: return build_cauchy(k, total, out);
    case 2: return build_jerasure_like(k, total, out);
    default: return ORC_INVALID_CUSTOM_MATRIX;
  }
}

/* ------------------------------------------------------------------------ */
/* Codec operations.                                                         */

/* src/core/encode.rs:532-602 (code_some_slices_with_outputs): parity row r is
 * the GF sum over inputs of M[k+r][j] * data[j]. */
void orc_classic_encode(size_t k, size_t m, const uint8_t *matrix,
                        const uint8_t *const *data, uint8_t *const *parity, size_t len) {
  gf8_init();
  for (size_t r = 0; r < m; r++) {
    const uint8_t *row = matrix + (k + r) * k;
    memset(parity[r], 0, len);
    for (size_t j = 0; j < k; j++) orc_gf8_mul_slice_xor(row[j], data[j], parity[r], len);
  }
}

/* src/core/verify.rs:14-33: re-encode into scratch and compare. */
int orc_classic_verify(size_t k, size_t m, const uint8_t *matrix,
                       const uint8_t *const *shards, size_t len) {
  uint8_t *scratch = (uint8_t *)malloc(m * len + 1);
  uint8_t **par = (uint8_t **)calloc(m + 1, sizeof(uint8_t *));
  for (size_t r = 0; r < m; r++) par[r] = scratch + r * len;
  orc_classic_encode(k, m, matrix, shards, par, len);
  int ok = 1;
  for (size_t r = 0; r < m && ok; r++) ok = memcmp(par[r], shards[k + r], len) == 0;
  free(par);
  free(scratch);
  return ok;
}

typedef struct {
  size_t survivors[256];
  size_t missing[256];
  size_t n_missing;
  size_t n_missing_data;
  size_t targets[256];
  size_t n_targets;
  size_t n_data_targets;
  int needs_inverse;
  int direct_parity;
  uint8_t *decode; /* k*k inverse of the selected survivor rows */
} plan_t;

/* src/core/recovery_plan.rs:262-298, 329-387, 425-517: survivors are the
 * first k present indices in ascending order; targets are the missing
 * indices (filtered by `required` for the Required goal); the inverse is
 * built only when some missing data shard contributes to a requested output. */
static int make_plan(size_t k, size_t m, const uint8_t *matrix, const uint8_t *present,
                     int goal, const uint8_t *required, size_t n_required, plan_t *p,
                     int *all_present) {
  size_t total = k + m;
  memset(p, 0, sizeof(*p));
  *all_present = 0;
  if (goal == 2 && n_required != k && n_required != total) return ORC_INVALID_SHARD_FLAGS;
  size_t n_present = 0, ns = 0;
  for (size_t i = 0; i < total; i++) {
    if (present[i]) {
      n_present++;
      if (ns < k) p->survivors[ns++] = i;
    } else {
      p->missing[p->n_missing++] = i;
      if (i < k) p->n_missing_data++;
    }
  }
  if (p->n_missing == 0) {
    *all_present = 1;
    return ORC_OK;
  }
  if (n_present < k) return ORC_TOO_FEW_SHARDS_PRESENT;
  for (size_t t = 0; t < p->n_missing; t++) {
    size_t idx = p->missing[t];
    int want;
    if (goal == 2)
      want = idx < n_required ? required[idx] != 0 : 0;
    else if (goal == 1)
      want = idx < k;
    else
      want = 1;
    if (!want) continue;
    p->targets[p->n_targets++] = idx;
    if (idx < k) p->n_data_targets++;
  }
  p->needs_inverse = p->n_missing_data > 0 && p->n_targets > 0;
  if (p->needs_inverse) {
    uint8_t *sel = (uint8_t *)malloc(k * k);
    p->decode = (uint8_t *)malloc(k * k);
    for (size_t r = 0; r < k; r++) memcpy(sel + r * k, matrix + p->survivors[r] * k, k);
    int rc = orc_gf8_invert(k, sel, p->decode);
    free(sel);
    if (rc != ORC_OK) {
      free(p->decode);
      p->decode = NULL;
      return ORC_INVALID_CUSTOM_MATRIX;
    }
  }
  p->direct_parity = goal == 2 && p->n_missing_data > 0 && p->n_targets > p->n_data_targets;
  return ORC_OK;
}

/* src/core/reconstruct.rs:318-416 (execute_classic_plan_with): the data stage
 * applies inverse rows to the survivors; the parity stage applies encoding
 * rows to the (present + recovered) data, or, for the Required goal with
 * missing data, composed rows over the survivors (recovery_plan.rs:480-515). */
int orc_classic_reconstruct(size_t k, size_t m, const uint8_t *matrix,
                            uint8_t *const *shards, const uint8_t *present, size_t len,
                            int goal, const uint8_t *required, size_t n_required) {
  gf8_init();
  plan_t p;
  int all_present;
  int rc = make_plan(k, m, matrix, present, goal, required, n_required, &p, &all_present);
  if (rc != ORC_OK || all_present) return rc;
  /* Data stage writes into scratch first so survivors are never clobbered. */
  uint8_t *rec = (uint8_t *)calloc(p.n_data_targets * len + 1, 1);
  for (size_t t = 0; t < p.n_data_targets; t++) {
    size_t d = p.targets[t];
    for (size_t c = 0; c < k; c++)
      orc_gf8_mul_slice_xor(p.decode[d * k + c], shards[p.survivors[c]], rec + t * len, len);
  }
  for (size_t t = 0; t < p.n_data_targets; t++) memcpy(shards[p.targets[t]], rec + t * len, len);
  free(rec);
  if (goal != 1) {
    for (size_t t = p.n_data_targets; t < p.n_targets; t++) {
      size_t pi = p.targets[t];
      const uint8_t *erow = matrix + pi * k;
      uint8_t *out = (uint8_t *)calloc(len + 1, 1);
      if (p.direct_parity) {
        for (size_t c = 0; c < k; c++) {
          size_t s = p.survivors[c];
          uint8_t co = s < k ? erow[s] : 0;
          for (size_t md = 0; md < p.n_missing; md++) {
            size_t d = p.missing[md];
            if (d >= k) break;
            co ^= MUL8[erow[d]][p.decode[d * k + c]];
          }
          orc_gf8_mul_slice_xor(co, shards[s], out, len);
        }
      } else {
        for (size_t j = 0; j < k; j++) orc_gf8_mul_slice_xor(erow[j], shards[j], out, len);
      }
      memcpy(shards[pi], out, len);
      free(out);
    }
  }
  free(p.decode);
  return ORC_OK;
}

/* Composed rows: data targets take inverse rows, parity targets take
 * E_p * Dec (equal to the two-stage result because every present data shard
 * is among the first k present shards). */
int orc_classic_recovery_rows(size_t k, size_t m, const uint8_t *matrix,
                              const uint8_t *present, int goal, const uint8_t *required,
                              size_t n_required, size_t *survivors, size_t *targets,
                              size_t *n_targets, uint8_t *rows) {
  gf8_init();
  plan_t p;
  int all_present;
  int rc = make_plan(k, m, matrix, present, goal, required, n_required, &p, &all_present);
  *n_targets = 0;
  if (rc != ORC_OK || all_present) return rc;
  size_t nt = goal == 1 ? p.n_data_targets : p.n_targets;
  memcpy(survivors, p.survivors, k * sizeof(size_t));
  memcpy(targets, p.targets, nt * sizeof(size_t));
  *n_targets = nt;
  for (size_t t = 0; t < nt; t++) {
    size_t idx = p.targets[t];
    uint8_t *row = rows + t * k;
    if (idx < k) {
      memcpy(row, p.decode + idx * k, k);
      continue;
    }
    const uint8_t *erow = matrix + idx * k;
    for (size_t c = 0; c < k; c++) {
      uint8_t co = 0;
      for (size_t j = 0; j < k; j++) {
        uint8_t dec;
        if (p.decode)
          dec = p.decode[j * k + c];
        else
          dec = p.survivors[c] == j ? 1 : 0;
        co ^= MUL8[erow[j]][dec];
      }
      row[c] = co;
    }
  }
  free(p.decode);
  return ORC_OK;
}

/* src/galois_8/policy.rs:543-700 (decode_idx) with the accumulation of
 * :79-140 (decode_idx_accumulate_reduced_outputs).  NULL entries of dst /
 * input stand for None.  With `expect` (n_expect flags), the first k expected
 * indices select the decoding inputs; each call adds, into every present
 * destination, the contributions of the inputs supplied in this call:
 * dst[o] ^= sum_j row_o[j] * input[valid[j]], where row_o is the inverse row
 * (data o < k) or the parity row times the inverse (parity o >= k) over the
 * selected columns.  Without `expect` (merge mode), dst[i] ^= input[i] for
 * every supplied input, after the whole layout has been validated.  The
 * checks run in the reference's order; an error leaves dst unchanged. */
int orc_classic_decode_idx(size_t k, size_t m, const uint8_t *matrix, uint8_t *const *dst,
                           const size_t *dst_lens, size_t n_dst, const uint8_t *expect, size_t n_expect,
                           const uint8_t *const *input, const size_t *input_lens, size_t n_input) {
  gf8_init();
  const size_t total = k + m;
  /* validate_opt_shard_count over [dst.len(), input.len()] (policy.rs:40-48) */
  const size_t counts[2] = {n_dst, n_input};
  for (int i = 0; i < 2; i++) {
    if (counts[i] < total) return ORC_TOO_FEW_SHARDS;
    if (counts[i] > total) return ORC_TOO_MANY_SHARDS;
  }
  if (!expect) {
    for (size_t i = 0; i < total; i++) {
      if (!input[i]) continue;
      if (!dst[i]) return ORC_TOO_FEW_SHARDS;
      if (dst_lens[i] != input_lens[i]) return ORC_INCORRECT_SHARD_SIZE;
    }
    for (size_t i = 0; i < total; i++)
      if (input[i])
        for (size_t b = 0; b < input_lens[i]; b++) dst[i][b] ^= input[i][b];
    return ORC_OK;
  }
  if (n_expect != total) return ORC_INVALID_SHARD_FLAGS;
  size_t valid[256], n_valid = 0;
  for (size_t i = 0; i < total; i++)
    if (expect[i]) valid[n_valid++] = i;
  if (n_valid < k) return ORC_TOO_FEW_SHARDS_PRESENT;
  /* shard_len: the first supplied buffer among the inputs, then the destinations */
  int have_len = 0;
  size_t len = 0;
  for (size_t i = 0; i < total && !have_len; i++)
    if (input[i]) len = input_lens[i], have_len = 1;
  for (size_t i = 0; i < total && !have_len; i++)
    if (dst[i]) len = dst_lens[i], have_len = 1;
  if (!have_len) return ORC_TOO_FEW_SHARDS_PRESENT;
  for (size_t i = 0; i < total; i++)
    if (input[i] && input_lens[i] != len) return ORC_INCORRECT_SHARD_SIZE;
  for (size_t i = 0; i < total; i++)
    if (dst[i] && dst_lens[i] != len) return ORC_INCORRECT_SHARD_SIZE;
  size_t outs[256], n_out = 0;
  for (size_t i = 0; i < total; i++)
    if (dst[i]) outs[n_out++] = i;
  if (n_out == 0) return ORC_OK;
  size_t pos[256], n_pos = 0;
  for (size_t c = 0; c < k; c++)
    if (input[valid[c]]) pos[n_pos++] = c;
  if (n_pos == 0) return ORC_OK;
  /* get_data_decode_matrix (src/core/reconstruct.rs:1176-1183) wants exactly k selected inputs */
  if (n_valid != k) return ORC_TOO_FEW_SHARDS_PRESENT;
  uint8_t *sel = (uint8_t *)malloc(k * k), *dec = (uint8_t *)malloc(k * k);
  for (size_t r = 0; r < k; r++) memcpy(sel + r * k, matrix + valid[r] * k, k);
  int rc = orc_gf8_invert(k, sel, dec);
  free(sel);
  if (rc != ORC_OK) {
    free(dec);
    return ORC_INVALID_CUSTOM_MATRIX;
  }
  if (len) {
    uint8_t *rows = (uint8_t *)malloc(n_out * n_pos);
    for (size_t o = 0; o < n_out; o++) {
      const size_t idx = outs[o];
      for (size_t j = 0; j < n_pos; j++) {
        const size_t col = pos[j];
        uint8_t v = 0;
        if (idx < k) {
          v = dec[idx * k + col];
        } else {
          const uint8_t *prow = matrix + idx * k;
          for (size_t i = 0; i < k; i++) v ^= MUL8[prow[i]][dec[i * k + col]];
        }
        rows[o * n_pos + j] = v;
      }
    }
    for (size_t o = 0; o < n_out; o++)
      for (size_t j = 0; j < n_pos; j++)
        orc_gf8_mul_slice_xor(rows[o * n_pos + j], input[valid[pos[j]]], dst[outs[o]], len);
    free(rows);
  }
  free(dec);
  return ORC_OK;
}
