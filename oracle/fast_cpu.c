/*
 * fast_cpu.c -- the timed CPU baseline.  TEST INFRASTRUCTURE ONLY (see
 * rs_oracle.h): this restates the reference's fastest x86 classic encode so
 * the benchmark can report a fair CPU number beside the GPU one.  It is never
 * part of the product path.
 *
 * It follows src/galois_8/x86/gfni_rows.rs:15-288 (each input vector is read
 * once per group of up to four outputs, with the output sums held in
 * registers) using GF2P8AFFINEQB when the host has GFNI
 * (src/galois_8/x86/gfni.rs:121-215, matrices derived as in
 * src/galois_8/mod.rs:9-33), at 64-byte width when the host also has
 * AVX-512 (the reference's first choice, src/galois_8/backend.rs:396-413,
 * dot_avx512 in gfni_rows.rs) and at 32-byte width otherwise, and the
 * split-nibble PSHUFB formulation of src/galois_8/x86/avx2.rs:85-155 without
 * GFNI.  Stripes are spread over threads the way the reference's rayon jobs
 * spread chunks (src/core/encode.rs:1177-1265).
 */
#include <immintrin.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

static int have_gfni(void) {
  __builtin_cpu_init();
  return __builtin_cpu_supports("gfni") && __builtin_cpu_supports("avx2");
}

static int have_gfni512(void) {
  __builtin_cpu_init();
  return have_gfni() && __builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw");
}

/* -1: the reference's own choice (widest GFNI the host has); otherwise a
 * forced kernel (2: GFNI at 64 bytes, 1: GFNI at 32 bytes, 0: nibble tables),
 * clamped to what the host supports. */
static int forced_kernel = -1;

static int selected_kernel(void) {
  const int best = have_gfni512() ? 2 : have_gfni() ? 1 : 0;
  return forced_kernel < 0 || forced_kernel > best ? best : forced_kernel;
}

void orc_fast_force_kernel(int kernel) { forced_kernel = kernel; }

int orc_fast_best_kernel(void) { return have_gfni512() ? 2 : have_gfni() ? 1 : 0; }

const char *orc_fast_kernel_name(void) {
  const int k = selected_kernel();
  return k == 2 ? "gfni-avx512-rows" : k == 1 ? "gfni-avx2-rows" : "avx2-nibble-rows";
}

static uint64_t gfni_matrix(uint8_t c) {
  uint64_t mtx = 0;
  for (int ib = 0; ib < 8; ib++) {
    uint8_t prod = orc_gf8_mul(c, (uint8_t)(1u << ib));
    for (int ob = 0; ob < 8; ob++)
      mtx |= (uint64_t)((prod >> ob) & 1) << ((7 - ob) * 8 + ib);
  }
  return mtx;
}

typedef struct {
  size_t k, m, len, n_stripes, next_stripe_stride, first;
  const uint8_t *matrix;
  uint8_t *const *ptrs;
  int gfni;      /* 2: GFNI at 64-byte width, 1: at 32-byte width, 0: nibble tables */
  size_t chunk;  /* columns per job: work is spread over (stripe, column chunk) */
} job_t;

__attribute__((target("avx2,gfni"))) static void rows_gfni(const job_t *j, uint8_t *const *sh, size_t x0, size_t len) {
  size_t k = j->k, m = j->m;
  for (size_t g = 0; g < m; g += 4) {
    size_t no = m - g < 4 ? m - g : 4;
    __m256i mats[4][256];
    for (size_t o = 0; o < no; o++)
      for (size_t i = 0; i < k; i++)
        mats[o][i] = _mm256_set1_epi64x((long long)gfni_matrix(j->matrix[(k + g + o) * k + i]));
    size_t x = x0;
    for (; x + 32 <= len; x += 32) {
      __m256i acc[4] = {_mm256_setzero_si256(), _mm256_setzero_si256(), _mm256_setzero_si256(),
                        _mm256_setzero_si256()};
      for (size_t i = 0; i < k; i++) {
        __m256i v = _mm256_loadu_si256((const __m256i *)(sh[i] + x));
        for (size_t o = 0; o < no; o++)
          acc[o] = _mm256_xor_si256(acc[o], _mm256_gf2p8affine_epi64_epi8(v, mats[o][i], 0));
      }
      for (size_t o = 0; o < no; o++) _mm256_storeu_si256((__m256i *)(sh[k + g + o] + x), acc[o]);
    }
    for (; x < len; x++)
      for (size_t o = 0; o < no; o++) {
        uint8_t a = 0;
        for (size_t i = 0; i < k; i++) a ^= orc_gf8_mul(j->matrix[(k + g + o) * k + i], sh[i][x]);
        sh[k + g + o][x] = a;
      }
  }
}

__attribute__((target("avx512f,avx512bw,gfni"))) static void rows_gfni512(const job_t *j, uint8_t *const *sh,
                                                                            size_t x0, size_t len) {
  size_t k = j->k, m = j->m;
  for (size_t g = 0; g < m; g += 4) {
    size_t no = m - g < 4 ? m - g : 4;
    __m512i mats[4][256];
    for (size_t o = 0; o < no; o++)
      for (size_t i = 0; i < k; i++)
        mats[o][i] = _mm512_set1_epi64((long long)gfni_matrix(j->matrix[(k + g + o) * k + i]));
    size_t x = x0;
    for (; x + 64 <= len; x += 64) {
      __m512i acc[4] = {_mm512_setzero_si512(), _mm512_setzero_si512(), _mm512_setzero_si512(),
                        _mm512_setzero_si512()};
      for (size_t i = 0; i < k; i++) {
        __m512i v = _mm512_loadu_si512((const void *)(sh[i] + x));
        for (size_t o = 0; o < no; o++)
          acc[o] = _mm512_xor_si512(acc[o], _mm512_gf2p8affine_epi64_epi8(v, mats[o][i], 0));
      }
      for (size_t o = 0; o < no; o++) _mm512_storeu_si512((void *)(sh[k + g + o] + x), acc[o]);
    }
    for (; x < len; x++)
      for (size_t o = 0; o < no; o++) {
        uint8_t a = 0;
        for (size_t i = 0; i < k; i++) a ^= orc_gf8_mul(j->matrix[(k + g + o) * k + i], sh[i][x]);
        sh[k + g + o][x] = a;
      }
  }
}

__attribute__((target("avx2"))) static void rows_nibble(const job_t *j, uint8_t *const *sh, size_t x0, size_t len) {
  size_t k = j->k, m = j->m;
  const __m256i mask = _mm256_set1_epi8(0x0f);
  for (size_t g = 0; g < m; g += 4) {
    size_t no = m - g < 4 ? m - g : 4;
    __m256i lo[4][256], hi[4][256];
    for (size_t o = 0; o < no; o++)
      for (size_t i = 0; i < k; i++) {
        uint8_t c = j->matrix[(k + g + o) * k + i];
        uint8_t tl[16], th[16];
        for (int n = 0; n < 16; n++) {
          tl[n] = orc_gf8_mul(c, (uint8_t)n);
          th[n] = orc_gf8_mul(c, (uint8_t)(n << 4));
        }
        __m128i a = _mm_loadu_si128((const __m128i *)tl), b = _mm_loadu_si128((const __m128i *)th);
        lo[o][i] = _mm256_broadcastsi128_si256(a);
        hi[o][i] = _mm256_broadcastsi128_si256(b);
      }
    size_t x = x0;
    for (; x + 32 <= len; x += 32) {
      __m256i acc[4] = {_mm256_setzero_si256(), _mm256_setzero_si256(), _mm256_setzero_si256(),
                        _mm256_setzero_si256()};
      for (size_t i = 0; i < k; i++) {
        __m256i v = _mm256_loadu_si256((const __m256i *)(sh[i] + x));
        __m256i vl = _mm256_and_si256(v, mask);
        __m256i vh = _mm256_and_si256(_mm256_srli_epi64(v, 4), mask);
        for (size_t o = 0; o < no; o++)
          acc[o] = _mm256_xor_si256(acc[o], _mm256_xor_si256(_mm256_shuffle_epi8(lo[o][i], vl),
                                                             _mm256_shuffle_epi8(hi[o][i], vh)));
      }
      for (size_t o = 0; o < no; o++) _mm256_storeu_si256((__m256i *)(sh[k + g + o] + x), acc[o]);
    }
    for (; x < len; x++)
      for (size_t o = 0; o < no; o++) {
        uint8_t a = 0;
        for (size_t i = 0; i < k; i++) a ^= orc_gf8_mul(j->matrix[(k + g + o) * k + i], sh[i][x]);
        sh[k + g + o][x] = a;
      }
  }
}

static void *worker(void *arg) {
  job_t *j = (job_t *)arg;
  size_t per = (j->len + j->chunk - 1) / j->chunk;
  for (size_t q = j->first; q < j->n_stripes * per; q += j->next_stripe_stride) {
    size_t s = q / per, c = q % per;
    size_t x0 = c * j->chunk, x1 = x0 + j->chunk < j->len ? x0 + j->chunk : j->len;
    uint8_t *const *sh = j->ptrs + s * (j->k + j->m);
    if (j->gfni == 2)
      rows_gfni512(j, sh, x0, x1);
    else if (j->gfni)
      rows_gfni(j, sh, x0, x1);
    else
      rows_nibble(j, sh, x0, x1);
  }
  return NULL;
}

int orc_fast_encode_batch(size_t k, size_t m, const uint8_t *matrix, uint8_t *const *shard_ptrs,
                          size_t n_stripes, size_t len, int threads) {
  if (k > 256 || threads < 1) return ORC_TOO_MANY_SHARDS;
  int gfni = selected_kernel();
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
  job_t *jobs = (job_t *)malloc(sizeof(job_t) * (size_t)threads);
  for (int t = 0; t < threads; t++) {
    size_t chunk = len / (size_t)threads + 1;
    if (n_stripes >= (size_t)threads || chunk < (64u << 10)) chunk = len > (256u << 10) ? (256u << 10) : len;
    chunk = (chunk + 31) & ~(size_t)31;
    job_t j = {k, m, len, n_stripes, (size_t)threads, (size_t)t, matrix, shard_ptrs, gfni, chunk};
    jobs[t] = j;
    pthread_create(&th[t], NULL, worker, &jobs[t]);
  }
  for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
  free(th);
  free(jobs);
  return ORC_OK;
}
