/*
 * cpu_port.c -- C restatement of the reference's runtime-dispatched x86 CPU
 * hot path, used ONLY as the timed CPU baseline (the reference is Rust and
 * cannot be built in this environment). TEST/BENCH INFRASTRUCTURE: nothing
 * in the product links it.
 *
 * It follows the reference's AVX2 + GFNI tier (backend `v3_gfni_crypto`):
 *   - Gf8D multiplies through VGF2P8AFFINEQB with one 8x8 GF(2) map per
 *     coefficient, byte r bit k = bit (7 - r) of c * x^k
 *     (src/kernel/tables.rs:172-213, src/kernel/x86/gf8.rs:239,805);
 *   - Gf8B multiplies through GF2P8MULB (src/kernel/x86/gf8.rs:44,735);
 *   - the blocked matrix kernel keeps 4 (then 2, then 1) destination rows in
 *     registers per 64-byte tile and folds every source term in before one
 *     store; overwrite seeds the accumulators with zero
 *     (src/kernel/x86/gf8.rs:2013-2070,2208-2315);
 *   - Gf16 uses the tower identity c*x = mul(x, same) ^ mul(swap16(x), cross)
 *     over GF2P8MULB (src/kernel/x86/gf16.rs:137-149,920-1068);
 *   - Gf32 composes per-row products from four byte permutations of each
 *     32-bit lane (the Klein group id/swap1/swap2/rev4,
 *     src/kernel/x86/gf32.rs:45-80,146).
 * Tails shorter than 32 bytes use the scalar oracle. The reference is
 * single-threaded; the multi-core figure runs independent jobs per thread.
 */
#pragma GCC target("avx2,gfni")
#include <immintrin.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <string.h>

#include "fgf_oracle.h"

typedef struct orc_job {
  int field;
  size_t k, m, row_len;
  const uint32_t *coeffs;     /* k x m term-major */
  const uint8_t *const *srcs; /* k */
  uint8_t *const *rows;       /* m */
  int overwrite;
} orc_job;

/* Callers check this before any other entry point: the whole file is compiled
 * for AVX2 + GFNI. */
int orc_port_supported(void) {
  __builtin_cpu_init();
  return __builtin_cpu_supports("avx2") && __builtin_cpu_supports("gfni");
}

/* ---------------------------------------------------------------- factors */

static uint64_t affine_map_8d(uint8_t c) {
  uint64_t map = 0;
  for (int r = 0; r < 8; ++r) {
    uint8_t row = 0;
    for (int k = 0; k < 8; ++k) {
      uint8_t col = (uint8_t)orc_mul(ORC_GF8D, c, 1u << k);
      row |= (uint8_t)(((col >> (7 - r)) & 1) << k);
    }
    map |= (uint64_t)row << (8 * r);
  }
  return map;
}

/* A prepared multiplier for one coefficient: up to four 256-bit factors. */
typedef struct {
  __m256i f[4];
} factor;

static factor prepare(int field, uint32_t c) {
  factor r;
  memset(&r, 0, sizeof r);
  if (field == ORC_GF8D) {
    r.f[0] = _mm256_set1_epi64x((long long)affine_map_8d((uint8_t)c));
  } else if (field == ORC_GF8B) {
    r.f[0] = _mm256_set1_epi8((char)c);
  } else if (field == ORC_GF16) {
    /* even byte: c0*a ^ 0x20 c1 * b ; odd byte: (c0^c1)*b ^ c1*a
       same = [c0, c0^c1], cross = [0x20 c1, c1] applied to swap16(x) */
    uint8_t c0 = (uint8_t)c, c1 = (uint8_t)(c >> 8);
    uint8_t d = (uint8_t)orc_mul(ORC_GF8B, 0x20, c1);
    r.f[0] = _mm256_set1_epi16((short)(c0 | ((c0 ^ c1) << 8)));
    r.f[1] = _mm256_set1_epi16((short)(d | (c1 << 8)));
  } else {
    /* Gf32: out byte q = XOR_s M[q][q ^ s] * x[q ^ s]; factor s holds
       M[q][q ^ s] in byte q of every 32-bit lane. M from the tower blocks. */
    uint16_t C0 = (uint16_t)c, C1 = (uint16_t)(c >> 16);
    uint16_t blk[2][2] = {{C0, (uint16_t)orc_mul(ORC_GF16, 0x2000, C1)}, {C1, (uint16_t)(C0 ^ C1)}};
    uint8_t M[4][4];
    for (int bi = 0; bi < 2; ++bi)
      for (int bj = 0; bj < 2; ++bj) {
        uint16_t x = blk[bi][bj];
        uint8_t x0 = (uint8_t)x, x1 = (uint8_t)(x >> 8);
        M[2 * bi][2 * bj] = x0;
        M[2 * bi][2 * bj + 1] = (uint8_t)orc_mul(ORC_GF8B, 0x20, x1);
        M[2 * bi + 1][2 * bj] = x1;
        M[2 * bi + 1][2 * bj + 1] = (uint8_t)(x0 ^ x1);
      }
    for (int s = 0; s < 4; ++s) {
      uint32_t lane = 0;
      for (int q = 0; q < 4; ++q) lane |= (uint32_t)M[q][q ^ s] << (8 * q);
      r.f[s] = _mm256_set1_epi32((int)lane);
    }
  }
  return r;
}

static inline __attribute__((always_inline)) __m256i mulv(int field, __m256i x, const factor *p) {
  if (field == ORC_GF8D) return _mm256_gf2p8affine_epi64_epi8(x, p->f[0], 0);
  if (field == ORC_GF8B) return _mm256_gf2p8mul_epi8(x, p->f[0]);
  if (field == ORC_GF16) {
    const __m256i sw = _mm256_setr_epi8(1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14, 1, 0, 3, 2, 5, 4, 7,
                                        6, 9, 8, 11, 10, 13, 12, 15, 14);
    return _mm256_xor_si256(_mm256_gf2p8mul_epi8(x, p->f[0]),
                            _mm256_gf2p8mul_epi8(_mm256_shuffle_epi8(x, sw), p->f[1]));
  }
  const __m256i s1 = _mm256_setr_epi8(1, 0, 3, 2, 5, 4, 7, 6, 9, 8, 11, 10, 13, 12, 15, 14, 1, 0, 3, 2, 5, 4, 7,
                                      6, 9, 8, 11, 10, 13, 12, 15, 14);
  const __m256i s2 = _mm256_setr_epi8(2, 3, 0, 1, 6, 7, 4, 5, 10, 11, 8, 9, 14, 15, 12, 13, 2, 3, 0, 1, 6, 7, 4,
                                      5, 10, 11, 8, 9, 14, 15, 12, 13);
  const __m256i s3 = _mm256_setr_epi8(3, 2, 1, 0, 7, 6, 5, 4, 11, 10, 9, 8, 15, 14, 13, 12, 3, 2, 1, 0, 7, 6, 5,
                                      4, 11, 10, 9, 8, 15, 14, 13, 12);
  __m256i r = _mm256_gf2p8mul_epi8(x, p->f[0]);
  r = _mm256_xor_si256(r, _mm256_gf2p8mul_epi8(_mm256_shuffle_epi8(x, s1), p->f[1]));
  r = _mm256_xor_si256(r, _mm256_gf2p8mul_epi8(_mm256_shuffle_epi8(x, s2), p->f[2]));
  r = _mm256_xor_si256(r, _mm256_gf2p8mul_epi8(_mm256_shuffle_epi8(x, s3), p->f[3]));
  return r;
}

/* ---------------------------------------------------------------- blocked kernel */

#define MAXFAC 1024 /* k * m coefficients handled by the blocked kernel */

/* Rows [g, g + R) of the job, R in {4, 2, 1}: 64-byte tiles, then 32-byte
 * steps, then the scalar tail. */
static inline __attribute__((always_inline)) void rows_block(const orc_job *J, const factor *fac, size_t g,
                                                             const int R, const int f) {
  const size_t L = J->row_len;
  size_t o = 0;
  for (; o + 64 <= L; o += 64) {
    __m256i acc[4][2];
    for (int r = 0; r < R; ++r)
      for (int h = 0; h < 2; ++h)
        acc[r][h] = J->overwrite ? _mm256_setzero_si256()
                                 : _mm256_loadu_si256((const __m256i *)(J->rows[g + r] + o + 32 * h));
    for (size_t t = 0; t < J->k; ++t) {
      const __m256i x0 = _mm256_loadu_si256((const __m256i *)(J->srcs[t] + o));
      const __m256i x1 = _mm256_loadu_si256((const __m256i *)(J->srcs[t] + o + 32));
      for (int r = 0; r < R; ++r) {
        const factor *p = &fac[t * J->m + g + r];
        acc[r][0] = _mm256_xor_si256(acc[r][0], mulv(f, x0, p));
        acc[r][1] = _mm256_xor_si256(acc[r][1], mulv(f, x1, p));
      }
    }
    for (int r = 0; r < R; ++r)
      for (int h = 0; h < 2; ++h) _mm256_storeu_si256((__m256i *)(J->rows[g + r] + o + 32 * h), acc[r][h]);
  }
  for (; o + 32 <= L; o += 32) {
    __m256i acc[4];
    for (int r = 0; r < R; ++r)
      acc[r] = J->overwrite ? _mm256_setzero_si256() : _mm256_loadu_si256((const __m256i *)(J->rows[g + r] + o));
    for (size_t t = 0; t < J->k; ++t) {
      const __m256i x = _mm256_loadu_si256((const __m256i *)(J->srcs[t] + o));
      for (int r = 0; r < R; ++r) acc[r] = _mm256_xor_si256(acc[r], mulv(f, x, &fac[t * J->m + g + r]));
    }
    for (int r = 0; r < R; ++r) _mm256_storeu_si256((__m256i *)(J->rows[g + r] + o), acc[r]);
  }
  if (o < L) {
    for (int r = 0; r < R; ++r) {
      uint8_t *row = J->rows[g + r] + o;
      if (J->overwrite) memset(row, 0, L - o);
      for (size_t t = 0; t < J->k; ++t) orc_mul_add(f, row, J->coeffs[t * J->m + g + r], J->srcs[t] + o, L - o);
    }
  }
}

/* One instantiation per (row group, field) so the accumulators live in
 * registers, as the reference's const-generic kernels do. */
#define ROWS_FN(R, F) \
  static __attribute__((noinline)) void rows_##R##_##F(const orc_job *J, const factor *fac, size_t g) { \
    rows_block(J, fac, g, R, F);                                                                          \
  }
ROWS_FN(4, 0) ROWS_FN(2, 0) ROWS_FN(1, 0)
ROWS_FN(4, 1) ROWS_FN(2, 1) ROWS_FN(1, 1)
ROWS_FN(4, 2) ROWS_FN(2, 2) ROWS_FN(1, 2)
ROWS_FN(4, 3) ROWS_FN(2, 3) ROWS_FN(1, 3)

typedef void (*rows_fn)(const orc_job *, const factor *, size_t);
static const rows_fn k_rows[4][3] = {{rows_4_0, rows_2_0, rows_1_0},
                                     {rows_4_1, rows_2_1, rows_1_1},
                                     {rows_4_2, rows_2_2, rows_1_2},
                                     {rows_4_3, rows_2_3, rows_1_3}};

static void run_job(const orc_job *J) {
  static __thread factor fac[MAXFAC];
  if (J->m == 0) return;
  if (J->k == 0 || J->k * J->m > MAXFAC) {
    /* outside the blocked kernel's limits: the scalar restatement */
    for (size_t j = 0; j < J->m; ++j) {
      if (J->overwrite) memset(J->rows[j], 0, J->row_len);
      for (size_t t = 0; t < J->k; ++t)
        orc_mul_add(J->field, J->rows[j], J->coeffs[t * J->m + j], J->srcs[t], J->row_len);
    }
    return;
  }
  for (size_t i = 0; i < J->k * J->m; ++i) fac[i] = prepare(J->field, J->coeffs[i]);
  const rows_fn *fn = k_rows[J->field & 3];
  size_t g = 0;
  for (; g + 4 <= J->m; g += 4) fn[0](J, fac, g);
  if (g + 2 <= J->m) {
    fn[1](J, fac, g);
    g += 2;
  }
  if (g < J->m) fn[2](J, fac, g);
}

typedef struct {
  const orc_job *jobs;
  size_t njobs;
  atomic_size_t next;
} pool_t;

static void *worker(void *arg) {
  pool_t *p = (pool_t *)arg;
  for (;;) {
    size_t i = atomic_fetch_add(&p->next, 1);
    if (i >= p->njobs) break;
    run_job(&p->jobs[i]);
  }
  return NULL;
}

/* Run every job (independent stripes) on `nthreads` threads. */
void orc_port_run_jobs(const orc_job *jobs, size_t njobs, int nthreads) {
  pool_t p;
  p.jobs = jobs;
  p.njobs = njobs;
  atomic_init(&p.next, 0);
  if (nthreads <= 1) {
    worker(&p);
    return;
  }
  pthread_t th[512];
  if (nthreads > 512) nthreads = 512;
  for (int i = 0; i < nthreads; ++i) pthread_create(&th[i], NULL, worker, &p);
  for (int i = 0; i < nthreads; ++i) pthread_join(th[i], NULL);
}

size_t orc_port_job_size(void) { return sizeof(orc_job); }
