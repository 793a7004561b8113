/*
 * leopard.c -- oracle restatement of the Leopard FFT codecs over GF(2^8) and
 * GF(2^16) from rustfs-erasure-codec 9.1.0 (src/core/leopard_gf8/,
 * src/core/leopard_gf16/).  TEST INFRASTRUCTURE ONLY (see rs_oracle.h).
 *
 * The loops restate the reference's plan builders and executors directly:
 * the encoder IFFT (mod.rs build_ifft_dit*_plan), the FFT
 * (build_fft_dit*_plan), the decoder IFFT (build_ifft_decode_dit*_plan), the
 * formal derivative and the FWHT error locator.  Every column of a shard is
 * independent, so the per-64-KiB chunking of the reference does not change a
 * byte and is not restated.
 */
#include <assert.h>
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

static size_t next_pow2(size_t n) {
  size_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

/* ======================================================================== */
/* GF(2^8) Leopard tables (src/core/leopard_gf8/tables.rs:8-145)              */

#define L8_ORDER 256
#define L8_MOD 255
static uint8_t L8_LOG[256], L8_EXP[256], L8_SKEW[255], L8_WALSH[256];
static uint8_t L8_MULV[256][256]; /* mul_luts[log_m].value */
static int l8_ready;

static uint8_t add_mod8(uint8_t a, uint8_t b) {
  unsigned s = (unsigned)a + b;
  return (uint8_t)(s + (s >> 8));
}
static uint8_t sub_mod8(uint8_t a, uint8_t b) {
  /* ops.rs:16-23: wrapping subtraction folded back into 8 bits. */
  unsigned long long d = (unsigned long long)a - (unsigned long long)b;
  return (uint8_t)(d + (d >> 8));
}
static uint8_t mul_log8_raw(uint8_t a, uint8_t log_b) {
  if (a == 0) return 0;
  return L8_EXP[add_mod8(L8_LOG[a], log_b)];
}

static void fwht2_8(uint8_t *a, uint8_t *b) {
  uint8_t s = add_mod8(*a, *b), d = sub_mod8(*a, *b);
  *a = s;
  *b = d;
}

/* ops.rs:26-58 / :60-93: radix-4 FWHT; `mtrunc` limits block starts. */
static void fwht8_mtrunc(uint8_t *data, size_t mtrunc) {
  size_t dist = 1, dist4 = 4;
  while (dist4 <= L8_ORDER) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      for (size_t off = r; off < r + dist; off++) {
        fwht2_8(&data[off], &data[off + dist]);
        fwht2_8(&data[off + 2 * dist], &data[off + 3 * dist]);
        fwht2_8(&data[off], &data[off + 2 * dist]);
        fwht2_8(&data[off + dist], &data[off + 3 * dist]);
      }
    }
    dist = dist4;
    dist4 <<= 2;
  }
}

static void l8_init(void) {
  if (l8_ready) return;
  static const uint8_t cantor[8] = {1, 214, 152, 146, 86, 200, 88, 230};
  unsigned state = 1;
  for (unsigned i = 0; i < L8_MOD; i++) {
    L8_EXP[state] = (uint8_t)i;
    state <<= 1;
    if (state >= L8_ORDER) state ^= 0x11D;
  }
  L8_EXP[0] = L8_MOD;
  L8_LOG[0] = 0;
  for (unsigned i = 0; i < 8; i++) {
    unsigned width = 1u << i;
    for (unsigned j = 0; j < width; j++) L8_LOG[j + width] = L8_LOG[j] ^ cantor[i];
  }
  for (unsigned i = 0; i < L8_ORDER; i++) L8_LOG[i] = L8_EXP[L8_LOG[i]];
  for (unsigned i = 0; i < L8_ORDER; i++) L8_EXP[L8_LOG[i]] = (uint8_t)i;
  L8_EXP[L8_MOD] = L8_EXP[0];

  /* init_fft_skew8 */
  uint8_t temp[7];
  for (unsigned i = 1; i < 8; i++) temp[i - 1] = (uint8_t)(1u << i);
  memset(L8_SKEW, 0, sizeof(L8_SKEW));
  for (unsigned m = 0; m < 7; m++) {
    size_t step = (size_t)1 << (m + 1);
    L8_SKEW[((size_t)1 << m) - 1] = 0;
    for (unsigned i = m; i < 7; i++) {
      size_t s = (size_t)1 << (i + 1);
      for (size_t j = ((size_t)1 << m) - 1; j < s; j += step) L8_SKEW[j + s] = L8_SKEW[j] ^ temp[i];
    }
    uint8_t prod = mul_log8_raw(temp[m], L8_LOG[temp[m] ^ 1]);
    temp[m] = (uint8_t)(L8_MOD - L8_LOG[prod]);
    for (unsigned i = m + 1; i < 7; i++) {
      uint8_t sum = add_mod8(L8_LOG[temp[i] ^ 1], temp[m]);
      temp[i] = mul_log8_raw(temp[i], sum);
    }
  }
  for (unsigned i = 0; i < L8_MOD; i++) L8_SKEW[i] = L8_LOG[L8_SKEW[i]];
  for (unsigned i = 0; i < L8_ORDER; i++) L8_WALSH[i] = L8_LOG[i];
  L8_WALSH[0] = 0;
  fwht8_mtrunc(L8_WALSH, L8_ORDER);

  /* init_mul8_lut: value[i] = tmp[i & 15] ^ tmp[(i >> 4) + 16]. */
  for (unsigned lm = 0; lm < 256; lm++) {
    uint8_t tmp[64];
    for (unsigned nib = 0, sh = 0; nib < 4; nib++, sh += 4)
      for (unsigned x = 0; x < 16; x++) tmp[nib * 16 + x] = mul_log8_raw((uint8_t)(x << sh), (uint8_t)lm);
    for (unsigned i = 0; i < 256; i++) L8_MULV[lm][i] = tmp[i & 15] ^ tmp[(i >> 4) + 16];
  }
  l8_ready = 1;
}

void orc_lgf8_tables(uint8_t *log_lut, uint8_t *exp_lut, uint8_t *fft_skew, uint8_t *log_walsh) {
  l8_init();
  memcpy(log_lut, L8_LOG, 256);
  memcpy(exp_lut, L8_EXP, 256);
  memcpy(fft_skew, L8_SKEW, 255);
  memcpy(log_walsh, L8_WALSH, 256);
}

uint8_t orc_lgf8_mul_log(uint8_t a, uint8_t log_b) {
  l8_init();
  return L8_MULV[log_b][a];
}

/* ops.rs:459-507: forward x ^= mul(y); y ^= x, inverse y ^= x; x ^= mul(y);
 * a multiplier log equal to the modulus means "only y ^= x". */
static void dit2_8(uint8_t *x, uint8_t *y, uint8_t lm, size_t len) {
  if (lm == L8_MOD) {
    for (size_t i = 0; i < len; i++) y[i] ^= x[i];
    return;
  }
  const uint8_t *t = L8_MULV[lm];
  for (size_t i = 0; i < len; i++) {
    x[i] ^= t[y[i]];
    y[i] ^= x[i];
  }
}
static void idit2_8(uint8_t *x, uint8_t *y, uint8_t lm, size_t len) {
  if (lm == L8_MOD) {
    for (size_t i = 0; i < len; i++) y[i] ^= x[i];
    return;
  }
  const uint8_t *t = L8_MULV[lm];
  for (size_t i = 0; i < len; i++) {
    y[i] ^= x[i];
    x[i] ^= t[y[i]];
  }
}

/* encode.rs dit4_at / dit4_pairwise: radix-4 block, falling back to the
 * pairs that exist when the last lane is past the work width. */
static void dit4_8(int forward, uint8_t **w, size_t nl, size_t a, size_t dist, uint8_t m01,
                   uint8_t m23, uint8_t m02, size_t len) {
  size_t b = a + dist, c = a + 2 * dist, d = a + 3 * dist;
  int ha = a < nl, hb = b < nl, hc = c < nl, hd = d < nl;
  if (forward) {
    if (ha && hc) dit2_8(w[a], w[c], m02, len);
    if (hb && hd) dit2_8(w[b], w[d], m02, len);
    if (ha && hb) dit2_8(w[a], w[b], m01, len);
    if (hc && hd) dit2_8(w[c], w[d], m23, len);
  } else {
    if (ha && hb) idit2_8(w[a], w[b], m01, len);
    if (hc && hd) idit2_8(w[c], w[d], m23, len);
    if (ha && hc) idit2_8(w[a], w[c], m02, len);
    if (hb && hd) idit2_8(w[b], w[d], m02, len);
  }
}

/* mod.rs build_ifft_dit8_plan + encode.rs ifft_dit_encoder8_with_plan:
 * `skew` is fft_skew offset by the group base; lanes >= mtrunc are zero. */
static void ifft_enc8(uint8_t **w, size_t mtrunc, size_t m, const uint8_t *skew,
                      size_t skew_len, size_t len) {
  size_t dist = 1, dist4 = 4;
  while (dist4 <= m) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      size_t iend = r + dist;
      assert(iend + 2 * dist < skew_len);
      uint8_t m01 = skew[iend], m02 = skew[iend + dist], m23 = skew[iend + 2 * dist];
      for (size_t i = r; i < iend; i++) dit4_8(0, w, m, i, dist, m01, m23, m02, len);
    }
    dist = dist4;
    dist4 <<= 2;
  }
  if (dist < m) {
    assert(dist < skew_len);
    uint8_t lm = skew[dist];
    for (size_t i = 0; i < dist; i++) idit2_8(w[i], w[i + dist], lm, len);
  }
}

/* mod.rs build_fft_dit8_plan (skew = full fft_skew, i_end - 1 indexing). */
static void fft8(uint8_t **w, size_t nl, size_t mtrunc, size_t m, size_t len) {
  size_t dist4 = m, dist = m >> 2;
  while (dist != 0) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      size_t iend = r + dist;
      uint8_t m01 = L8_SKEW[iend - 1], m02 = L8_SKEW[iend + dist - 1],
              m23 = L8_SKEW[iend + 2 * dist - 1];
      for (size_t i = r; i < iend; i++) dit4_8(1, w, nl, i, dist, m01, m23, m02, len);
    }
    dist4 = dist;
    dist >>= 2;
  }
  if (dist4 == 2)
    for (size_t r = 0; r < mtrunc; r += 2)
      if (r + 1 < nl) dit2_8(w[r], w[r + 1], L8_SKEW[r], len);
}

/* mod.rs build_ifft_decode_dit8_plan + decode.rs ifft_dit_decode8_with_plan. */
static void ifft_dec8(uint8_t **w, size_t mtrunc, size_t n, size_t len) {
  size_t dist = 1, dist4 = 4;
  if (dist4 <= n) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      size_t avail = mtrunc - r < 4 ? mtrunc - r : 4;
      for (size_t s = r + avail; s < r + 4; s++)
        if (s < n) memset(w[s], 0, len);
      size_t iend = r + dist;
      dit4_8(0, w, n, r, dist, L8_SKEW[iend - 1], L8_SKEW[iend + 2 * dist - 1],
             L8_SKEW[iend + dist - 1], len);
    }
    for (size_t s = (mtrunc + 3) & ~(size_t)3; s < n; s++) memset(w[s], 0, len);
    dist = dist4;
    dist4 <<= 2;
    while (dist4 <= n) {
      for (size_t r = 0; r < mtrunc; r += dist4) {
        size_t iend = r + dist;
        uint8_t m01 = L8_SKEW[iend - 1], m02 = L8_SKEW[iend + dist - 1],
                m23 = L8_SKEW[iend + 2 * dist - 1];
        for (size_t i = r; i < iend; i++) dit4_8(0, w, n, i, dist, m01, m23, m02, len);
      }
      dist = dist4;
      dist4 <<= 2;
    }
  } else {
    for (size_t s = mtrunc; s < n; s++) memset(w[s], 0, len);
  }
  if (dist < n) {
    uint8_t lm = L8_SKEW[dist - 1];
    for (size_t i = 0; i < dist; i++)
      if (i + dist < n) idit2_8(w[i], w[i + dist], lm, len);
  }
}

/* decode.rs compute_formal_derivative: lower ^= higher. */
static void formal_derivative8(uint8_t **w, size_t n, size_t len) {
  for (size_t i = 1; i < n; i++) {
    size_t width = ((i ^ (i - 1)) + 1) >> 1;
    for (size_t j = 0; j < width; j++) {
      size_t lo = i - width + j, hi = i + j;
      if (hi < n && lo < n)
        for (size_t x = 0; x < len; x++) w[lo][x] ^= w[hi][x];
    }
  }
}

static int leopard_combo_fits(size_t k, size_t p, size_t order) {
  size_t m = next_pow2(p);
  if (k == 0 || p == 0 || m > order) return 0;
  size_t rounded = (k + m - 1) / m * m;
  return rounded <= (order > m ? order - m : 0);
}

/* driver.rs:18-52 + encode.rs:194-372. */
int orc_lgf8_encode(size_t k, size_t p, const uint8_t *const *data, uint8_t *const *parity,
                    size_t len) {
  l8_init();
  if (len == 0 || len % 64) return ORC_INCORRECT_SHARD_SIZE;
  if (!leopard_combo_fits(k, p, 256)) return ORC_TOO_MANY_SHARDS;
  size_t m = next_pow2(p);
  if (m > L8_MOD) return ORC_TOO_MANY_SHARDS;
  size_t mtrunc = k < m ? k : m, last = k % m;
  uint8_t *buf = (uint8_t *)calloc(2 * m * len, 1);
  uint8_t **w = (uint8_t **)malloc(2 * m * sizeof(uint8_t *));
  for (size_t i = 0; i < 2 * m; i++) w[i] = buf + i * len;
  const uint8_t *skew = L8_SKEW + (m - 1);
  size_t skew_len = L8_MOD - (m - 1);
  for (size_t i = 0; i < mtrunc; i++) memcpy(w[i], data[i], len);
  ifft_enc8(w, mtrunc, m, skew, skew_len, len);
  if (m < k) {
    size_t g = m, so = m;
    for (; g + m <= k; g += m, so += m) {
      for (size_t i = 0; i < m; i++) memcpy(w[m + i], data[g + i], len);
      ifft_enc8(w + m, m, m, skew + so, skew_len - so, len);
      for (size_t i = 0; i < m; i++)
        for (size_t x = 0; x < len; x++) w[i][x] ^= w[m + i][x];
    }
    if (last) {
      for (size_t i = 0; i < m; i++) {
        if (i < last)
          memcpy(w[m + i], data[g + i], len);
        else
          memset(w[m + i], 0, len);
      }
      ifft_enc8(w + m, last, m, skew + so, skew_len - so, len);
      for (size_t i = 0; i < m; i++)
        for (size_t x = 0; x < len; x++) w[i][x] ^= w[m + i][x];
    }
  }
  fft8(w, m, p, m, len);
  for (size_t i = 0; i < p; i++) memcpy(parity[i], w[i], len);
  free(w);
  free(buf);
  return ORC_OK;
}

/* decode.rs:58-113 (compute_error_locs). */
void orc_lgf8_error_locators(size_t k, size_t p, const uint8_t *present, uint8_t *err) {
  l8_init();
  size_t m = next_pow2(p), work_size = m + k;
  memset(err, 0, 256);
  for (size_t i = 0; i < p; i++) err[i] = present[k + i] ? 0 : 1;
  for (size_t i = p; i < m; i++) err[i] = 1;
  for (size_t i = 0; i < k; i++) err[m + i] = present[i] ? 0 : 1;
  fwht8_mtrunc(err, work_size);
  for (size_t i = 0; i < 256; i++)
    if (err[i]) err[i] = (uint8_t)(((unsigned)err[i] * L8_WALSH[i]) % L8_MOD);
  fwht8_mtrunc(err, 256);
}

/* decode.rs:291-420 (reconstruct_with_resources).  `want` selects which
 * missing shards receive output bytes. */
int orc_lgf8_reconstruct(size_t k, size_t p, uint8_t *const *shards, const uint8_t *present,
                         const uint8_t *want, size_t len) {
  l8_init();
  size_t total = k + p, np = 0, nmiss = 0;
  for (size_t i = 0; i < total; i++) np += present[i] ? 1 : 0;
  nmiss = total - np;
  if (np < k) return ORC_TOO_FEW_SHARDS_PRESENT;
  if (len == 0 || len % 64) return ORC_INCORRECT_SHARD_SIZE;
  if (nmiss == 0) return ORC_OK;
  if (nmiss > p) return ORC_TOO_FEW_SHARDS_PRESENT;
  size_t m = next_pow2(p);
  if (m > L8_MOD) return ORC_TOO_MANY_SHARDS;
  size_t work_size = m + k;
  if (work_size > 256) return ORC_TOO_MANY_SHARDS;
  size_t n = next_pow2(work_size);
  uint8_t err[256];
  orc_lgf8_error_locators(k, p, present, err);
  size_t input_count = m;
  for (size_t i = 0; i < k; i++)
    if (present[i]) input_count = m + i + 1;
  uint8_t *buf = (uint8_t *)calloc(n * len, 1);
  uint8_t **w = (uint8_t **)malloc(n * sizeof(uint8_t *));
  for (size_t i = 0; i < n; i++) w[i] = buf + i * len;
  for (size_t i = 0; i < k; i++)
    if (present[i]) {
      const uint8_t *t = L8_MULV[err[m + i]];
      for (size_t x = 0; x < len; x++) w[m + i][x] = t[shards[i][x]];
    }
  for (size_t i = 0; i < p; i++)
    if (present[k + i]) {
      const uint8_t *t = L8_MULV[err[i]];
      for (size_t x = 0; x < len; x++) w[i][x] = t[shards[k + i][x]];
    }
  ifft_dec8(w, input_count, n, len);
  formal_derivative8(w, n, len);
  fft8(w, n, work_size, n, len);
  for (size_t i = 0; i < total; i++) {
    if (present[i] || !want[i]) continue;
    size_t lane = i >= k ? i - k : m + i;
    const uint8_t *t = L8_MULV[(uint8_t)(L8_MOD - err[lane])];
    for (size_t x = 0; x < len; x++) shards[i][x] = t[w[lane][x]];
  }
  free(w);
  free(buf);
  return ORC_OK;
}

/* ======================================================================== */
/* GF(2^16) Leopard (src/core/leopard_gf16/)                                */

#define L16_ORDER 65536
#define L16_MOD 65535
static uint16_t *L16_LOG, *L16_EXP, *L16_SKEW, *L16_WALSH;
static int l16_ready;

static uint16_t add_mod16(uint16_t a, uint16_t b) {
  uint32_t s = (uint32_t)a + b;
  return (uint16_t)(s + (s >> 16));
}
static uint16_t sub_mod16(uint16_t a, uint16_t b) {
  uint32_t d = (uint32_t)a - (uint32_t)b;
  return (uint16_t)(d + (d >> 16));
}
/* ops.rs:12-23 */
static uint16_t mul_log16(uint16_t a, uint16_t log_b) {
  if (a == 0) return 0;
  return L16_EXP[add_mod16(L16_LOG[a], log_b)];
}

static void fwht2_16(uint16_t *a, uint16_t *b) {
  uint16_t s = add_mod16(*a, *b), d = sub_mod16(*a, *b);
  *a = s;
  *b = d;
}

/* ops.rs:264-362: fwht16 / fwht16_mtrunc / fwht16_variable all reduce to the
 * same radix-4 butterflies for a 65,536-point input. */
static void fwht16_mtrunc(uint16_t *data, size_t order, size_t mtrunc) {
  size_t dist = 1, dist4 = 4;
  while (dist4 <= order) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      for (size_t off = r; off < r + dist; off++) {
        fwht2_16(&data[off], &data[off + dist]);
        fwht2_16(&data[off + 2 * dist], &data[off + 3 * dist]);
        fwht2_16(&data[off], &data[off + 2 * dist]);
        fwht2_16(&data[off + dist], &data[off + 3 * dist]);
      }
    }
    dist = dist4;
    dist4 <<= 2;
  }
}

static void l16_init(void) {
  if (l16_ready) return;
  static const uint16_t cantor[16] = {0x0001, 0xACCA, 0x3C0E, 0x163E, 0xC582, 0xED2E,
                                      0x914C, 0x4012, 0x6C98, 0x10D8, 0x6A72, 0xB900,
                                      0xFDB8, 0xFB34, 0xFF38, 0x991E};
  L16_LOG = (uint16_t *)calloc(L16_ORDER, 2);
  L16_EXP = (uint16_t *)calloc(2 * L16_ORDER, 2);
  L16_SKEW = (uint16_t *)calloc(L16_MOD, 2);
  L16_WALSH = (uint16_t *)calloc(L16_ORDER, 2);
  /* tables.rs:22-62 */
  uint32_t state = 1;
  for (uint32_t i = 0; i < L16_MOD; i++) {
    L16_EXP[state] = (uint16_t)i;
    state <<= 1;
    if (state >= L16_ORDER) state ^= 0x1002D;
  }
  L16_EXP[0] = L16_MOD;
  L16_LOG[0] = 0;
  for (unsigned i = 0; i < 16; i++) {
    uint32_t width = 1u << i;
    for (uint32_t j = 0; j < width; j++) L16_LOG[j + width] = L16_LOG[j] ^ cantor[i];
  }
  for (uint32_t i = 0; i < L16_ORDER; i++) L16_LOG[i] = L16_EXP[L16_LOG[i]];
  for (uint32_t i = 0; i < L16_ORDER; i++) L16_EXP[L16_LOG[i]] = (uint16_t)i;
  L16_EXP[L16_MOD] = L16_EXP[0];

  /* tables.rs:64-116 (init_fft_skew16) */
  uint16_t temp[15];
  for (unsigned i = 1; i < 16; i++) temp[i - 1] = (uint16_t)(1u << i);
  for (unsigned m = 0; m < 15; m++) {
    size_t step = (size_t)1 << (m + 1);
    L16_SKEW[((size_t)1 << m) - 1] = 0;
    for (unsigned i = m; i < 15; i++) {
      size_t s = (size_t)1 << (i + 1);
      for (size_t j = ((size_t)1 << m) - 1; j < s; j += step) L16_SKEW[j + s] = L16_SKEW[j] ^ temp[i];
    }
    uint16_t prod = mul_log16(temp[m], L16_LOG[temp[m] ^ 1]);
    temp[m] = (uint16_t)(L16_MOD - (uint32_t)L16_LOG[prod]);
    for (unsigned i = m + 1; i < 15; i++) {
      uint16_t sum = add_mod16(L16_LOG[temp[i] ^ 1], temp[m]);
      temp[i] = mul_log16(temp[i], sum);
    }
  }
  for (uint32_t i = 0; i < L16_MOD; i++) L16_SKEW[i] = L16_LOG[L16_SKEW[i]];
  for (uint32_t i = 0; i < L16_ORDER; i++) L16_WALSH[i] = L16_LOG[i];
  L16_WALSH[0] = 0;
  fwht16_mtrunc(L16_WALSH, L16_ORDER, L16_ORDER);
  l16_ready = 1;
}

void orc_lgf16_tables(uint16_t *log_lut, uint16_t *exp_lut, uint16_t *fft_skew,
                      uint16_t *log_walsh) {
  l16_init();
  memcpy(log_lut, L16_LOG, L16_ORDER * 2);
  memcpy(exp_lut, L16_EXP, 2 * L16_ORDER * 2);
  memcpy(fft_skew, L16_SKEW, L16_MOD * 2);
  memcpy(log_walsh, L16_WALSH, L16_ORDER * 2);
}

uint16_t orc_lgf16_mul_log(uint16_t a, uint16_t log_b) {
  l16_init();
  return mul_log16(a, log_b);
}

/* ops.rs:375-447 */
static void dit2_16(uint16_t *x, uint16_t *y, uint16_t lm, size_t len) {
  if (lm == L16_MOD) {
    for (size_t i = 0; i < len; i++) y[i] ^= x[i];
    return;
  }
  for (size_t i = 0; i < len; i++) {
    x[i] ^= mul_log16(y[i], lm);
    y[i] ^= x[i];
  }
}
static void idit2_16(uint16_t *x, uint16_t *y, uint16_t lm, size_t len) {
  if (lm == L16_MOD) {
    for (size_t i = 0; i < len; i++) y[i] ^= x[i];
    return;
  }
  for (size_t i = 0; i < len; i++) {
    y[i] ^= x[i];
    x[i] ^= mul_log16(y[i], lm);
  }
}

static void dit4_16(int forward, uint16_t **w, size_t nl, size_t a, size_t dist, uint16_t m01,
                    uint16_t m23, uint16_t m02, size_t len) {
  size_t b = a + dist, c = a + 2 * dist, d = a + 3 * dist;
  int ha = a < nl, hb = b < nl, hc = c < nl, hd = d < nl;
  if (forward) {
    if (ha && hc) dit2_16(w[a], w[c], m02, len);
    if (hb && hd) dit2_16(w[b], w[d], m02, len);
    if (ha && hb) dit2_16(w[a], w[b], m01, len);
    if (hc && hd) dit2_16(w[c], w[d], m23, len);
  } else {
    if (ha && hb) idit2_16(w[a], w[b], m01, len);
    if (hc && hd) idit2_16(w[c], w[d], m23, len);
    if (ha && hc) idit2_16(w[a], w[c], m02, len);
    if (hb && hd) idit2_16(w[b], w[d], m02, len);
  }
}

static void ifft_enc16(uint16_t **w, size_t mtrunc, size_t m, const uint16_t *skew,
                       size_t skew_len, size_t len) {
  size_t dist = 1, dist4 = 4;
  while (dist4 <= m) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      size_t iend = r + dist;
      assert(iend + 2 * dist < skew_len);
      uint16_t m01 = skew[iend], m02 = skew[iend + dist], m23 = skew[iend + 2 * dist];
      for (size_t i = r; i < iend; i++) dit4_16(0, w, m, i, dist, m01, m23, m02, len);
    }
    dist = dist4;
    dist4 <<= 2;
  }
  if (dist < m) {
    assert(dist < skew_len);
    uint16_t lm = skew[dist];
    for (size_t i = 0; i < dist; i++) idit2_16(w[i], w[i + dist], lm, len);
  }
}

static void fft16(uint16_t **w, size_t nl, size_t mtrunc, size_t m, size_t len) {
  size_t dist4 = m, dist = m >> 2;
  while (dist != 0) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      size_t iend = r + dist;
      uint16_t m01 = L16_SKEW[iend - 1], m02 = L16_SKEW[iend + dist - 1],
               m23 = L16_SKEW[iend + 2 * dist - 1];
      for (size_t i = r; i < iend; i++) dit4_16(1, w, nl, i, dist, m01, m23, m02, len);
    }
    dist4 = dist;
    dist >>= 2;
  }
  if (dist4 == 2)
    for (size_t r = 0; r < mtrunc; r += 2)
      if (r + 1 < nl) dit2_16(w[r], w[r + 1], L16_SKEW[r], len);
}

static void ifft_dec16(uint16_t **w, size_t mtrunc, size_t n, size_t len) {
  size_t dist = 1, dist4 = 4;
  if (dist4 <= n) {
    for (size_t r = 0; r < mtrunc; r += dist4) {
      size_t avail = mtrunc - r < 4 ? mtrunc - r : 4;
      for (size_t s = r + avail; s < r + 4; s++)
        if (s < n) memset(w[s], 0, len * 2);
      size_t iend = r + dist;
      dit4_16(0, w, n, r, dist, L16_SKEW[iend - 1], L16_SKEW[iend + 2 * dist - 1],
              L16_SKEW[iend + dist - 1], len);
    }
    for (size_t s = (mtrunc + 3) & ~(size_t)3; s < n; s++) memset(w[s], 0, len * 2);
    dist = dist4;
    dist4 <<= 2;
    while (dist4 <= n) {
      for (size_t r = 0; r < mtrunc; r += dist4) {
        size_t iend = r + dist;
        uint16_t m01 = L16_SKEW[iend - 1], m02 = L16_SKEW[iend + dist - 1],
                 m23 = L16_SKEW[iend + 2 * dist - 1];
        for (size_t i = r; i < iend; i++) dit4_16(0, w, n, i, dist, m01, m23, m02, len);
      }
      dist = dist4;
      dist4 <<= 2;
    }
  } else {
    for (size_t s = mtrunc; s < n; s++) memset(w[s], 0, len * 2);
  }
  if (dist < n) {
    uint16_t lm = L16_SKEW[dist - 1];
    for (size_t i = 0; i < dist; i++)
      if (i + dist < n) idit2_16(w[i], w[i + dist], lm, len);
  }
}

static void formal_derivative16(uint16_t **w, size_t n, size_t len) {
  for (size_t i = 1; i < n; i++) {
    size_t width = ((i ^ (i - 1)) + 1) >> 1;
    for (size_t j = 0; j < width; j++) {
      size_t lo = i - width + j, hi = i + j;
      if (hi < n && lo < n)
        for (size_t x = 0; x < len; x++) w[lo][x] ^= w[hi][x];
    }
  }
}

/* ops.rs:513-807: element i of a 64-byte block is byte[i] | byte[i+32] << 8. */
static void user_to_work16(const uint8_t *src, uint16_t *dst, size_t bytes) {
  for (size_t blk = 0; blk < bytes; blk += 64)
    for (size_t i = 0; i < 32; i++)
      dst[blk / 2 + i] = (uint16_t)(src[blk + i] | ((uint16_t)src[blk + i + 32] << 8));
}
static void work_to_user16(const uint16_t *src, uint8_t *dst, size_t bytes) {
  for (size_t blk = 0; blk < bytes; blk += 64)
    for (size_t i = 0; i < 32; i++) {
      dst[blk + i] = (uint8_t)src[blk / 2 + i];
      dst[blk + i + 32] = (uint8_t)(src[blk / 2 + i] >> 8);
    }
}

/* driver.rs:6-30 + encode.rs:109-252. */
int orc_lgf16_encode(size_t k, size_t p, const uint8_t *const *data, uint8_t *const *parity,
                     size_t len) {
  l16_init();
  if (len == 0 || len % 64) return ORC_INCORRECT_SHARD_SIZE;
  if (!leopard_combo_fits(k, p, 65536)) return ORC_TOO_MANY_SHARDS;
  size_t m = next_pow2(p);
  if (m > L16_MOD) return ORC_TOO_MANY_SHARDS;
  size_t el = len / 2;
  size_t mtrunc = k < m ? k : m, last = k % m;
  uint16_t *buf = (uint16_t *)calloc(2 * m * el, 2);
  uint16_t **w = (uint16_t **)malloc(2 * m * sizeof(uint16_t *));
  for (size_t i = 0; i < 2 * m; i++) w[i] = buf + i * el;
  const uint16_t *skew = L16_SKEW + (m - 1);
  size_t skew_len = L16_MOD - (m - 1);
  for (size_t i = 0; i < mtrunc; i++) user_to_work16(data[i], w[i], len);
  ifft_enc16(w, mtrunc, m, skew, skew_len, el);
  if (m < k) {
    size_t g = m, so = m;
    for (; g + m <= k; g += m, so += m) {
      for (size_t i = 0; i < m; i++) user_to_work16(data[g + i], w[m + i], len);
      ifft_enc16(w + m, m, m, skew + so, skew_len - so, el);
      for (size_t i = 0; i < m; i++)
        for (size_t x = 0; x < el; x++) w[i][x] ^= w[m + i][x];
    }
    if (last) {
      for (size_t i = 0; i < m; i++) {
        if (i < last)
          user_to_work16(data[g + i], w[m + i], len);
        else
          memset(w[m + i], 0, el * 2);
      }
      ifft_enc16(w + m, last, m, skew + so, skew_len - so, el);
      for (size_t i = 0; i < m; i++)
        for (size_t x = 0; x < el; x++) w[i][x] ^= w[m + i][x];
    }
  }
  fft16(w, m, p, m, el);
  for (size_t i = 0; i < p; i++) work_to_user16(w[i], parity[i], len);
  free(w);
  free(buf);
  return ORC_OK;
}

/* decode.rs:177-216 (compute_error_locs16). */
void orc_lgf16_error_locators(size_t k, size_t p, const uint8_t *present, uint16_t *err) {
  l16_init();
  size_t m = next_pow2(p), work_size = m + k;
  memset(err, 0, L16_ORDER * 2);
  for (size_t i = 0; i < p; i++)
    if (!present[k + i]) err[i] = 1;
  for (size_t i = p; i < m; i++) err[i] = 1;
  for (size_t i = 0; i < k; i++)
    if (!present[i]) err[m + i] = 1;
  fwht16_mtrunc(err, L16_ORDER, work_size);
  for (size_t i = 0; i < L16_ORDER; i++)
    if (err[i]) err[i] = (uint16_t)(((uint64_t)err[i] * L16_WALSH[i]) % L16_MOD);
  fwht16_mtrunc(err, L16_ORDER, L16_ORDER);
}

/* decode.rs:704-910. */
int orc_lgf16_reconstruct(size_t k, size_t p, uint8_t *const *shards, const uint8_t *present,
                          const uint8_t *want, size_t len) {
  l16_init();
  size_t total = k + p, np = 0;
  for (size_t i = 0; i < total; i++) np += present[i] ? 1 : 0;
  if (np < k) return ORC_TOO_FEW_SHARDS_PRESENT;
  if (len == 0 || len % 64) return ORC_INCORRECT_SHARD_SIZE;
  size_t nmiss = total - np;
  if (nmiss == 0) return ORC_OK;
  size_t m = next_pow2(p);
  if (m > L16_MOD) return ORC_TOO_MANY_SHARDS;
  size_t work_size = m + k;
  if (work_size > L16_ORDER) return ORC_TOO_MANY_SHARDS;
  size_t n = next_pow2(work_size);
  if (nmiss > p) return ORC_TOO_FEW_SHARDS_PRESENT;
  uint16_t *err = (uint16_t *)malloc(L16_ORDER * 2);
  orc_lgf16_error_locators(k, p, present, err);
  size_t input_count = m;
  for (size_t i = 0; i < k; i++)
    if (present[i]) input_count = m + i + 1;
  size_t el = len / 2;
  uint16_t *buf = (uint16_t *)calloc(n * el, 2);
  uint16_t **w = (uint16_t **)malloc(n * sizeof(uint16_t *));
  for (size_t i = 0; i < n; i++) w[i] = buf + i * el;
  for (size_t i = 0; i < k; i++)
    if (present[i]) {
      user_to_work16(shards[i], w[m + i], len);
      for (size_t x = 0; x < el; x++) w[m + i][x] = mul_log16(w[m + i][x], err[m + i]);
    }
  for (size_t i = 0; i < p; i++)
    if (present[k + i]) {
      user_to_work16(shards[k + i], w[i], len);
      for (size_t x = 0; x < el; x++) w[i][x] = mul_log16(w[i][x], err[i]);
    }
  ifft_dec16(w, input_count, n, el);
  formal_derivative16(w, n, el);
  fft16(w, n, work_size, n, el);
  uint16_t *tmp = (uint16_t *)malloc(el * 2);
  for (size_t i = 0; i < total; i++) {
    if (present[i] || !want[i]) continue;
    size_t lane = i >= k ? i - k : m + i;
    uint16_t inv = (uint16_t)(L16_MOD - err[lane]);
    for (size_t x = 0; x < el; x++) tmp[x] = mul_log16(w[lane][x], inv);
    work_to_user16(tmp, shards[i], len);
  }
  free(tmp);
  free(w);
  free(buf);
  free(err);
  return ORC_OK;
}
