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

void build_compact_tables(int field, const uint32_t* coeffs, size_t m, size_t t0, size_t k,
                          size_t g0, size_t G, uint32_t* out) {
  const int E = field_bytes(field);
  const int R = 4 / E;
  for (size_t tt = 0; tt < k; ++tt) {
    const size_t t = t0 + tt;
    for (size_t g = 0; g < G; ++g) {
      // Images of the R coefficients this group covers (rows past m
      // contribute zero products).
      uint32_t img[4][4][8];
      for (int r = 0; r < R; ++r) {
        const size_t j = (g0 + g) * R + r;
        if (j < m) {
          coeff_images(field, coeffs[t * m + j], img[r]);
        } else {
          std::memset(img[r], 0, sizeof img[r]);
        }
      }
      for (int p = 0; p < E; ++p) {
        uint32_t* slot = out + ((tt * E + p) * G + g) * kCompactWords;
        for (int half = 0; half < 2; ++half)
          for (int n = 0; n < 16; ++n) {
            const uint8_t x = static_cast<uint8_t>(half ? (n << 4) : n);
            uint32_t word = 0;
            for (int q = 0; q < 4; ++q)
              word |= static_cast<uint32_t>(image_byte(img[q / E], p, x, q % E)) << (8 * q);
            slot[half * 16 + n] = word;
          }
      }
    }
  }
}

}  // namespace fgfc
