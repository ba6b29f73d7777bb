/*
 * fgf_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see fgf_oracle.h).
 *
 * Restates, in plain scalar C, the reference library's:
 *   - flat GF(2^8) arithmetic: shift/XOR product (src/field/flat8.rs:105-122),
 *     LOG/EXP tables from the generator (flat8.rs:382-410), table product
 *     (flat8.rs:147-156), inverse with inv(0)=0 (flat8.rs:171-180),
 *     division with x/0=0 (flat8.rs:188-193); polynomials and generators
 *     0x11B/0x03 (src/field/gf8b.rs:57) and 0x11D/0x02 (src/field/gf8d.rs:40);
 *   - GF(2^16) tower a+b*u, u^2+u+0x20 over Gf8B, Karatsuba product and
 *     conjugate/norm inverse (src/field/gf16.rs:54-60,143-180);
 *   - GF(2^32) tower over GF(2^16), DELTA 0x2000 (src/field/gf32.rs:36-42,121-150);
 *   - GF(2^64) tower over GF(2^32), DELTA 0x20000000 (src/field/gf64.rs:1-11,120-151);
 *   - the canonical Fan-Paar towers at 8, 16, 32 and 64 bits
 *     (src/field/fan_paar.rs:1-14,66-150);
 *   - elementwise op semantics including the zero/one shortcuts
 *     (src/kernel/scalar.rs:20-130, src/ops.rs:342-941).
 */
#include "fgf_oracle.h"

#include <string.h>

/* ---------------------------------------------------------------- GF(2^8) */

static uint8_t g_exp[2][255];
static uint8_t g_log[2][256];
static int g_ready = 0;

static const uint8_t k_low[2] = {0x1B, 0x1D};  /* 0x11B, 0x11D minus x^8 */
static const uint8_t k_gen[2] = {0x03, 0x02};

static uint8_t gf8_xtime_mul(int which, uint8_t a, uint8_t b) {
  /* flat8.rs:105-122: for each bit of b, accumulate a, then a *= x. */
  uint8_t acc = 0;
  for (int i = 0; i < 8; ++i) {
    if ((b >> i) & 1) acc ^= a;
    uint8_t carry = (uint8_t)(a & 0x80);
    a = (uint8_t)(a << 1);
    if (carry) a ^= k_low[which];
  }
  return acc;
}

static void gf8_init(void) {
  if (g_ready) return;
  for (int w = 0; w < 2; ++w) {
    uint8_t v = 1;
    for (int i = 0; i < 255; ++i) {
      g_exp[w][i] = v;
      v = gf8_xtime_mul(w, v, k_gen[w]);
    }
    memset(g_log[w], 0, 256);
    for (int i = 0; i < 255; ++i) g_log[w][g_exp[w][i]] = (uint8_t)i;
  }
  g_ready = 1;
}

static uint8_t gf8_mul(int w, uint8_t a, uint8_t b) {
  if (a == 0 || b == 0) return 0;
  gf8_init();
  return g_exp[w][((unsigned)g_log[w][a] + g_log[w][b]) % 255];
}

static uint8_t gf8_inv(int w, uint8_t a) {
  if (a == 0) return 0;
  gf8_init();
  return g_exp[w][(255u - g_log[w][a]) % 255];
}

/* ---------------------------------------------------------------- towers */

static uint16_t gf16_mul(uint16_t x, uint16_t y) {
  uint8_t a = (uint8_t)x, b = (uint8_t)(x >> 8), c = (uint8_t)y, d = (uint8_t)(y >> 8);
  uint8_t ac = gf8_mul(0, a, c), bd = gf8_mul(0, b, d);
  uint8_t lo = (uint8_t)(ac ^ gf8_mul(0, 0x20, bd));
  uint8_t hi = (uint8_t)(gf8_mul(0, (uint8_t)(a ^ b), (uint8_t)(c ^ d)) ^ ac);
  return (uint16_t)(lo | (hi << 8));
}

static uint16_t gf16_inv(uint16_t x) {
  uint8_t a = (uint8_t)x, b = (uint8_t)(x >> 8);
  if (x == 0) return 0;
  uint8_t norm = (uint8_t)(gf8_mul(0, a, a) ^ gf8_mul(0, a, b) ^ gf8_mul(0, 0x20, gf8_mul(0, b, b)));
  uint8_t ni = gf8_inv(0, norm);
  return (uint16_t)(gf8_mul(0, (uint8_t)(a ^ b), ni) | (gf8_mul(0, b, ni) << 8));
}

static uint32_t gf32_mul(uint32_t x, uint32_t y) {
  uint16_t a = (uint16_t)x, b = (uint16_t)(x >> 16), c = (uint16_t)y, d = (uint16_t)(y >> 16);
  uint16_t ac = gf16_mul(a, c), bd = gf16_mul(b, d);
  uint16_t lo = (uint16_t)(ac ^ gf16_mul(0x2000, bd));
  uint16_t hi = (uint16_t)(gf16_mul((uint16_t)(a ^ b), (uint16_t)(c ^ d)) ^ ac);
  return (uint32_t)lo | ((uint32_t)hi << 16);
}

static uint32_t gf32_inv(uint32_t x) {
  uint16_t a = (uint16_t)x, b = (uint16_t)(x >> 16);
  if (x == 0) return 0;
  uint16_t norm = (uint16_t)(gf16_mul(a, a) ^ gf16_mul(a, b) ^ gf16_mul(0x2000, gf16_mul(b, b)));
  uint16_t ni = gf16_inv(norm);
  return (uint32_t)gf16_mul((uint16_t)(a ^ b), ni) | ((uint32_t)gf16_mul(b, ni) << 16);
}

/* ---------------------------------------------------------------- Fan-Paar towers */
/*
 * Canonical Fan-Paar binary tower (src/field/fan_paar.rs:1-14,66-150): each
 * level of 2h bits is the quadratic extension X^2 + alpha*X + 1 of the h-bit
 * level, alpha being that level's own top generator; an element is
 * lo + hi*X with lo in the low h bits. Products recurse by Karatsuba down to
 * one bit (fan_paar.rs:80-94); multiplying by alpha is the linear recurrence
 * of fan_paar.rs:67-76; inversion is conjugate times inverse norm
 * (fan_paar.rs:137-148).
 */
static uint64_t fp_low(unsigned bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1ull); }

static uint64_t fp_mul_alpha(uint64_t v, unsigned bits) {
  if (bits == 1) return v & 1u;
  unsigned h = bits / 2;
  uint64_t a0 = v & fp_low(h), a1 = v >> h;
  return a1 | ((a0 ^ fp_mul_alpha(a1, h)) << h);
}

static uint64_t fp_mul_bits(uint64_t x, uint64_t y, unsigned bits) {
  if (bits == 1) return x & y & 1u;
  unsigned h = bits / 2;
  uint64_t m = fp_low(h);
  uint64_t a0 = x & m, a1 = x >> h, b0 = y & m, b1 = y >> h;
  uint64_t z0 = fp_mul_bits(a0, b0, h), z2 = fp_mul_bits(a1, b1, h);
  uint64_t z1 = fp_mul_bits(a0 ^ a1, b0 ^ b1, h) ^ z0 ^ z2;
  return (z0 ^ z2) | ((z1 ^ fp_mul_alpha(z2, h)) << h);
}

static uint64_t fp_inv_bits(uint64_t x, unsigned bits) {
  if (bits == 1) return x & 1u;
  unsigned h = bits / 2;
  uint64_t a0 = x & fp_low(h), a1 = x >> h;
  uint64_t a0z1 = a0 ^ fp_mul_alpha(a1, h);
  uint64_t norm = fp_mul_bits(a0, a0z1, h) ^ fp_mul_bits(a1, a1, h);
  uint64_t ni = fp_inv_bits(norm, h);
  return fp_mul_bits(ni, a0z1, h) | (fp_mul_bits(ni, a1, h) << h);
}

static unsigned fp_bits(int field) {
  return field == ORC_FP8 ? 8u : (field == ORC_FP16 ? 16u : (field == ORC_FP32 ? 32u : 64u));
}

/* GF(2^64) = GF(2^32)[w]/(w^2 + w + 0x20000000), a + b*w with a in the low
 * half (src/field/gf64.rs:1-11,120-151): the same Karatsuba product and
 * conjugate / norm inverse as one level down. */
static uint64_t gf64_mul(uint64_t x, uint64_t y) {
  uint32_t a = (uint32_t)x, b = (uint32_t)(x >> 32), c = (uint32_t)y, d = (uint32_t)(y >> 32);
  uint32_t ac = gf32_mul(a, c), bd = gf32_mul(b, d);
  uint32_t lo = ac ^ gf32_mul(0x20000000u, bd);
  uint32_t hi = gf32_mul(a ^ b, c ^ d) ^ ac;
  return (uint64_t)lo | ((uint64_t)hi << 32);
}

static uint64_t gf64_inv(uint64_t x) {
  uint32_t a = (uint32_t)x, b = (uint32_t)(x >> 32);
  if (x == 0) return 0;
  uint32_t norm = gf32_mul(a, a) ^ gf32_mul(a, b) ^ gf32_mul(0x20000000u, gf32_mul(b, b));
  uint32_t ni = gf32_inv(norm);
  return (uint64_t)gf32_mul(a ^ b, ni) | ((uint64_t)gf32_mul(b, ni) << 32);
}

/* ---------------------------------------------------------------- public scalar API */

int orc_bytes(int field) {
  switch (field) {
    case ORC_GF8B:
    case ORC_GF8D: return 1;
    case ORC_GF16: return 2;
    case ORC_GF32: return 4;
    case ORC_FP8: return 1;
    case ORC_FP16: return 2;
    case ORC_FP32: return 4;
    case ORC_GF64:
    case ORC_FP64: return 8;
    default: return 0;
  }
}

uint32_t orc_mul(int field, uint32_t a, uint32_t b) {
  switch (field) {
    case ORC_GF8B: return gf8_mul(0, (uint8_t)a, (uint8_t)b);
    case ORC_GF8D: return gf8_mul(1, (uint8_t)a, (uint8_t)b);
    case ORC_GF16: return gf16_mul((uint16_t)a, (uint16_t)b);
    case ORC_GF32: return gf32_mul(a, b);
    case ORC_FP8:
    case ORC_FP16:
    case ORC_FP32: {
      unsigned bits = fp_bits(field);
      return (uint32_t)fp_mul_bits(a & fp_low(bits), b & fp_low(bits), bits);
    }
    default: return 0;
  }
}

uint32_t orc_mul_xtime(int field, uint32_t a, uint32_t b) {
  if (field == ORC_GF8B) return gf8_xtime_mul(0, (uint8_t)a, (uint8_t)b);
  if (field == ORC_GF8D) return gf8_xtime_mul(1, (uint8_t)a, (uint8_t)b);
  return orc_mul(field, a, b);
}

uint32_t orc_inv(int field, uint32_t a) {
  switch (field) {
    case ORC_GF8B: return gf8_inv(0, (uint8_t)a);
    case ORC_GF8D: return gf8_inv(1, (uint8_t)a);
    case ORC_GF16: return gf16_inv((uint16_t)a);
    case ORC_GF32: return gf32_inv(a);
    case ORC_FP8:
    case ORC_FP16:
    case ORC_FP32: {
      unsigned bits = fp_bits(field);
      return (uint32_t)fp_inv_bits(a & fp_low(bits), bits);
    }
    default: return 0;
  }
}

uint32_t orc_inv_xtime(int field, uint32_t a) {
  /* flat8.rs:126-143: a^254 by square-and-multiply over the bits of 254. */
  if (field != ORC_GF8B && field != ORC_GF8D) return orc_inv(field, a);
  if (a == 0) return 0;
  uint32_t r = 1;
  for (int i = 0; i < 8; ++i) {
    r = orc_mul_xtime(field, r, r);
    if ((254u >> (7 - i)) & 1) r = orc_mul_xtime(field, r, a);
  }
  return r;
}

uint32_t orc_div(int field, uint32_t a, uint32_t b) {
  if (a == 0 || b == 0) return 0;
  return orc_mul(field, a, orc_inv(field, b));
}

uint32_t orc_square(int field, uint32_t a) { return orc_mul(field, a, a); }

uint32_t orc_pow(int field, uint32_t a, uint64_t e) {
  uint32_t base = a, r = 1;
  while (e) {
    if (e & 1) r = orc_mul(field, r, base);
    base = orc_mul(field, base, base);
    e >>= 1;
  }
  return r;
}

uint64_t orc_mul64(int field, uint64_t a, uint64_t b) {
  if (field == ORC_GF64) return gf64_mul(a, b);
  if (field == ORC_FP64) return fp_mul_bits(a, b, 64);
  return orc_mul(field, (uint32_t)a, (uint32_t)b);
}

uint64_t orc_inv64(int field, uint64_t a) {
  if (field == ORC_GF64) return gf64_inv(a);
  if (field == ORC_FP64) return fp_inv_bits(a, 64);
  return orc_inv(field, (uint32_t)a);
}

uint64_t orc_pow64(int field, uint64_t a, uint64_t e) {
  uint64_t base = a, r = 1;
  while (e) {
    if (e & 1) r = orc_mul64(field, r, base);
    base = orc_mul64(field, base, base);
    e >>= 1;
  }
  return r;
}

void orc_noise(uint8_t *out, size_t len, uint64_t seed) {
  uint64_t s = seed | 1u;
  for (size_t i = 0; i < len; ++i) {
    s = s * 6364136223846793005ull + 1ull;
    out[i] = (uint8_t)(s >> 33);
  }
}

/* ---------------------------------------------------------------- element I/O */

static uint64_t rd(int field, const uint8_t *p) {
  int n = orc_bytes(field);
  uint64_t v = 0;
  for (int i = 0; i < n; ++i) v |= (uint64_t)p[i] << (8 * i);
  return v;
}

static void wr(int field, uint8_t *p, uint64_t v) {
  int n = orc_bytes(field);
  for (int i = 0; i < n; ++i) p[i] = (uint8_t)(v >> (8 * i));
}

/* ---------------------------------------------------------------- ops */

void orc_xor(uint8_t *dst, const uint8_t *src, size_t len) {
  for (size_t i = 0; i < len; ++i) dst[i] ^= src[i];
}

void orc_mul_add(int field, uint8_t *dst, uint64_t coeff, const uint8_t *src, size_t len) {
  /* scalar.rs:40-57: zero is a no-op, one is XOR, otherwise per element. */
  if (coeff == 0) return;
  if (coeff == 1) { orc_xor(dst, src, len); return; }
  int b = orc_bytes(field);
  for (size_t i = 0; i + b <= len; i += b)
    wr(field, dst + i, rd(field, dst + i) ^ orc_mul64(field, rd(field, src + i), coeff));
}

void orc_mul_into(int field, uint8_t *dst, uint64_t coeff, const uint8_t *src, size_t len) {
  /* ops.rs:381-392 */
  if (coeff == 0) { memset(dst, 0, len); return; }
  if (coeff == 1) { memmove(dst, src, len); return; }
  int b = orc_bytes(field);
  for (size_t i = 0; i + b <= len; i += b) wr(field, dst + i, orc_mul64(field, rd(field, src + i), coeff));
}

void orc_mul_assign(int field, uint8_t *dst, uint64_t coeff, size_t len) {
  /* scalar.rs:60-72 */
  if (coeff == 1) return;
  if (coeff == 0) { memset(dst, 0, len); return; }
  int b = orc_bytes(field);
  for (size_t i = 0; i + b <= len; i += b) wr(field, dst + i, orc_mul64(field, rd(field, dst + i), coeff));
}

void orc_mul_elementwise(int field, uint8_t *dst, const uint8_t *a, const uint8_t *bb, size_t len) {
  /* scalar.rs:119-130 */
  int b = orc_bytes(field);
  for (size_t i = 0; i + b <= len; i += b) wr(field, dst + i, orc_mul64(field, rd(field, a + i), rd(field, bb + i)));
}

void orc_mul_add_scatter(int field, uint8_t *rows, size_t row_len, const uint64_t *coeffs,
                         size_t nrows, const uint8_t *src) {
  /* scalar.rs:75-79: one mul_add per row. */
  for (size_t j = 0; j < nrows; ++j) orc_mul_add(field, rows + j * row_len, coeffs[j], src, row_len);
}

void orc_mul_add_gather(int field, uint8_t *dst, size_t len, const uint64_t *coeffs,
                        const uint8_t *const *srcs, size_t nsrcs) {
  /* scalar.rs:112-116 */
  for (size_t t = 0; t < nsrcs; ++t) orc_mul_add(field, dst, coeffs[t], srcs[t], len);
}

void orc_dot_product(int field, uint8_t *dst, size_t len, const uint64_t *coeffs,
                     const uint8_t *const *srcs, size_t nsrcs) {
  /* ops.rs:597-624: overwrite; empty or all-zero fills zero. */
  memset(dst, 0, len);
  orc_mul_add_gather(field, dst, len, coeffs, srcs, nsrcs);
}

void orc_mul_add_matrix(int field, uint8_t *rows, size_t row_len, size_t nrows,
                        const uint64_t *coeffs, const uint8_t *const *srcs, size_t nsrcs) {
  /* scalar.rs:82-94: every term applied to every row. */
  for (size_t t = 0; t < nsrcs; ++t)
    for (size_t j = 0; j < nrows; ++j)
      orc_mul_add(field, rows + j * row_len, coeffs[t * nrows + j], srcs[t], row_len);
}

void orc_dot_product_matrix(int field, uint8_t *rows, size_t row_len, size_t nrows,
                            const uint64_t *coeffs, const uint8_t *const *srcs, size_t nsrcs) {
  /* ops.rs:773-810 / kernel/mod.rs:507-533: zero the used rows, accumulate. */
  memset(rows, 0, row_len * nrows);
  orc_mul_add_matrix(field, rows, row_len, nrows, coeffs, srcs, nsrcs);
}

void orc_mul_add_matrix_scattered(int field, uint8_t *dst, size_t row_len,
                                  const size_t *row_starts, size_t nrows,
                                  const uint64_t *coeffs, const uint8_t *const *srcs,
                                  size_t nsrcs) {
  /* scalar.rs:98-109 */
  for (size_t t = 0; t < nsrcs; ++t)
    for (size_t j = 0; j < nrows; ++j)
      orc_mul_add(field, dst + row_starts[j], coeffs[t * nrows + j], srcs[t], row_len);
}

/* ---------------------------------------------------------------- RS recipes */

void orc_cauchy(int field, uint32_t *c, size_t m, size_t k, uint32_t x0) {
  for (size_t i = 0; i < m; ++i)
    for (size_t j = 0; j < k; ++j) c[i * k + j] = orc_inv(field, (uint32_t)(x0 + i) ^ (uint32_t)j);
}

int orc_invert(int field, uint32_t *a, size_t n) {
  /* Augment with the identity in a scratch copy (n <= 64 here). */
  uint32_t aug[64 * 128];
  if (n > 64) return -1;
  size_t w = 2 * n;
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < w; ++j)
      aug[i * w + j] = j < n ? a[i * n + j] : (j - n == i ? 1u : 0u);
  for (size_t col = 0; col < n; ++col) {
    size_t piv = col;
    while (piv < n && aug[piv * w + col] == 0) ++piv;
    if (piv == n) return -1;
    if (piv != col)
      for (size_t j = 0; j < w; ++j) {
        uint32_t t = aug[piv * w + j];
        aug[piv * w + j] = aug[col * w + j];
        aug[col * w + j] = t;
      }
    uint32_t pinv = orc_inv(field, aug[col * w + col]);
    for (size_t j = 0; j < w; ++j) aug[col * w + j] = orc_mul(field, aug[col * w + j], pinv);
    for (size_t i = 0; i < n; ++i) {
      if (i == col) continue;
      uint32_t f = aug[i * w + col];
      if (f == 0) continue;
      for (size_t j = 0; j < w; ++j) aug[i * w + j] ^= orc_mul(field, f, aug[col * w + j]);
    }
  }
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j) a[i * n + j] = aug[i * w + n + j];
  return 0;
}

static uint32_t gen_entry(const uint32_t *c, size_t k, size_t row, size_t col) {
  /* Systematic generator [I_k ; C]. */
  if (row < k) return row == col ? 1u : 0u;
  return c[(row - k) * k + col];
}

int orc_decode_matrix(int field, const uint32_t *c, size_t k, size_t m,
                      const size_t *survivors, const size_t *erased, size_t r, uint32_t *out) {
  uint32_t sub[64 * 64];
  (void)m;
  if (k > 64) return -1;
  for (size_t i = 0; i < k; ++i)
    for (size_t j = 0; j < k; ++j) sub[i * k + j] = gen_entry(c, k, survivors[i], j);
  if (orc_invert(field, sub, k) != 0) return -1;
  for (size_t e = 0; e < r; ++e)
    for (size_t t = 0; t < k; ++t) {
      uint32_t acc = 0;
      for (size_t q = 0; q < k; ++q)
        acc ^= orc_mul(field, gen_entry(c, k, erased[e], q), sub[q * k + t]);
      out[e * k + t] = acc;
    }
  return 0;
}
