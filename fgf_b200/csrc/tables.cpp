// tables.cpp -- host derivation of the compact nibble tables a launch uploads.
#include <cstring>

#include "internal.hpp"

namespace fgfc {

const Gf8Log& gf8b_tab() {
  static const Gf8Log t(0x1B, 0x03);
  return t;
}
const Gf8Log& gf8d_tab() {
  static const Gf8Log t(0x1D, 0x02);
  return t;
}

void build_compact_tables(int field, const uint64_t* coeffs, size_t m, size_t t0, size_t k,
                          size_t g0, size_t G, uint32_t* out) {
  const int E = field_bytes(field);
  for (size_t tt = 0; tt < k; ++tt) {
    const size_t t = t0 + tt;
    for (size_t g = 0; g < G; ++g) {
      // The group's 4 output bytes are the flat output bytes
      // f = 4 (g0 + g) + q of the m * E (row f / E, byte f % E); rows past m
      // contribute zero products. Images per row this group touches.
      uint64_t img[4][8][8];
      size_t row[4];
      int ri[4], ob[4];
      int nr = 0;
      for (int q = 0; q < 4; ++q) {
        const size_t f = 4 * (g0 + g) + q;
        const size_t j = f / E;
        ob[q] = static_cast<int>(f % E);
        ri[q] = -1;
        if (j >= m) continue;
        for (int r = 0; r < nr; ++r)
          if (row[r] == j) ri[q] = r;
        if (ri[q] < 0) {
          row[nr] = j;
          coeff_images(field, coeffs[t * m + j], img[nr]);
          ri[q] = nr++;
        }
      }
      for (int p = 0; p < E; ++p) {
        uint32_t* slot = out + ((tt * E + p) * G + g) * kCompactWords;
        for (int half = 0; half < 2; ++half)
          for (int n = 0; n < 16; ++n) {
            const uint8_t x = static_cast<uint8_t>(half ? (n << 4) : n);
            uint32_t word = 0;
            for (int q = 0; q < 4; ++q)
              if (ri[q] >= 0) word |= static_cast<uint32_t>(image_byte(img[ri[q]], p, x, ob[q])) << (8 * q);
            slot[half * 16 + n] = word;
          }
      }
    }
  }
}

namespace {

// c * x over the 4-byte base field of an 8-byte field.
uint32_t wide_half_mul(int field, uint32_t c, uint32_t x) {
  return field == kGf64 ? gf32_mul(c, x) : static_cast<uint32_t>(fp_mul(c, x, 32));
}

// Nibble tables of a GF(2)-linear map on 32-bit words, given the images of
// its 32 input bits: table p (input byte p) at out + p * 32.
void linear_tables(const uint32_t img[32], uint32_t* out, size_t stride_slots) {
  for (int p = 0; p < 4; ++p) {
    uint32_t* slot = out + p * stride_slots * kCompactWords;
    for (int half = 0; half < 2; ++half)
      for (int n = 0; n < 16; ++n) {
        uint32_t v = 0;
        for (int b = 0; b < 4; ++b)
          if ((n >> b) & 1) v ^= img[8 * p + 4 * half + b];
        slot[half * 16 + n] = v;
      }
  }
}

}  // namespace

void build_wide_tables(int field, const uint64_t* coeffs, size_t m, size_t t0, size_t k, size_t j0, size_t M,
                       uint32_t* out) {
  for (size_t tt = 0; tt < k; ++tt)
    for (size_t j = 0; j < M; ++j) {
      const uint64_t c = coeffs[(t0 + tt) * m + j0 + j];
      const uint32_t c0 = static_cast<uint32_t>(c), c1 = static_cast<uint32_t>(c >> 32);
      const uint32_t cp[3] = {c0, c1, c0 ^ c1};
      for (int P = 0; P < 3; ++P) {
        uint32_t img[32];
        for (int i = 0; i < 32; ++i) img[i] = wide_half_mul(field, cp[P], 1u << i);
        // slot of (tt, P, p = 0, j); input byte p is M slots further on
        linear_tables(img, out + ((tt * 3 + P) * 4 * M + j) * kCompactWords, M);
      }
    }
}

void build_wide_fixup(int field, uint32_t* out) {
  uint32_t img[32];
  for (int i = 0; i < 32; ++i) {
    const uint32_t v = 1u << i;
    img[i] = field == kGf64 ? gf32_mul(0x20000000u, v) : v ^ static_cast<uint32_t>(fp_mul_alpha(v, 32));
  }
  linear_tables(img, out, 1);
}

void build_kara16_tables(const uint64_t* coeffs, size_t m, size_t k, size_t Gq, uint32_t* out) {
  for (size_t t = 0; t < k; ++t)
    for (int P = 0; P < 3; ++P)
      for (size_t q = 0; q < Gq; ++q) {
        uint8_t cp[4];
        for (int r = 0; r < 4; ++r) {
          const size_t j = 4 * q + r;
          const uint64_t c = j < m ? coeffs[t * m + j] : 0;
          const uint8_t c0 = static_cast<uint8_t>(c), c1 = static_cast<uint8_t>(c >> 8);
          cp[r] = P == 0 ? c0 : P == 1 ? c1 : static_cast<uint8_t>(c0 ^ c1);
        }
        uint32_t* slot = out + ((t * 3 + P) * Gq + q) * kCompactWords;
        for (int half = 0; half < 2; ++half)
          for (int n = 0; n < 16; ++n) {
            const uint8_t x = static_cast<uint8_t>(half ? (n << 4) : n);
            uint32_t w = 0;
            for (int r = 0; r < 4; ++r) w |= static_cast<uint32_t>(gf8b_mul(cp[r], x)) << (8 * r);
            slot[half * 16 + n] = w;
          }
      }
}

}  // namespace fgfc
