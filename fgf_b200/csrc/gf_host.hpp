// gf_host.hpp -- host-side field arithmetic used to derive device tables and
// decode matrices. Product code (independent of the oracle under oracle/).
//
// Field definitions follow the reference crate:
//   Gf8B: GF(2)[x]/(x^8+x^4+x^3+x+1), generator 0x03     (src/field/gf8b.rs:57)
//   Gf8D: GF(2)[x]/(x^8+x^4+x^3+x^2+1), generator 0x02   (src/field/gf8d.rs:40)
//   Gf16: Gf8B[u]/(u^2+u+0x20), element a + b*u stored [a, b]  (src/field/gf16.rs:54-60)
//   Gf32: Gf16[v]/(v^2+v+0x2000), element a + b*v stored LE    (src/field/gf32.rs:36-42)
// inv(0) = 0 and x/0 = 0 by convention (src/field/mod.rs:38-41).
#pragma once
#include <cstddef>
#include <cstdint>

namespace fgfc {

enum Field : int { kGf8B = 0, kGf8D = 1, kGf16 = 2, kGf32 = 3 };

inline int field_bytes(int f) { return f == kGf16 ? 2 : (f == kGf32 ? 4 : ((f == kGf8B || f == kGf8D) ? 1 : 0)); }
inline const char* field_name(int f) {
  switch (f) {
    case kGf8B: return "GF(2^8)";
    case kGf8D: return "GF(2^8)/0x11D";
    case kGf16: return "GF(2^16)";
    case kGf32: return "GF(2^32)";
    default: return "?";
  }
}
inline uint32_t field_mask(int f) { return f == kGf32 ? 0xFFFFFFFFu : (f == kGf16 ? 0xFFFFu : 0xFFu); }

// Log/antilog tables for one flat GF(2^8), built from the generator by
// repeated carry-less doubling with reduction.
struct Gf8Log {
  uint8_t exp[512];
  uint8_t log[256];
  explicit Gf8Log(uint8_t low, uint8_t gen) {
    uint8_t v = 1;
    for (int i = 0; i < 255; ++i) {
      exp[i] = v;
      // v *= gen by shift-and-add over the bits of gen
      uint8_t a = v, acc = 0;
      for (int b = 0; b < 8; ++b) {
        if ((gen >> b) & 1) acc ^= a;
        a = static_cast<uint8_t>((a << 1) ^ ((a & 0x80) ? low : 0));
      }
      v = acc;
    }
    for (int i = 255; i < 512; ++i) exp[i] = exp[i - 255];
    log[0] = 0;
    for (int i = 0; i < 255; ++i) log[exp[i]] = static_cast<uint8_t>(i);
  }
  uint8_t mul(uint8_t a, uint8_t b) const { return (a && b) ? exp[log[a] + log[b]] : 0; }
  uint8_t inv(uint8_t a) const { return a ? exp[255 - log[a]] : 0; }
};

const Gf8Log& gf8b_tab();
const Gf8Log& gf8d_tab();

inline uint8_t gf8b_mul(uint8_t a, uint8_t b) { return gf8b_tab().mul(a, b); }

inline uint16_t gf16_mul(uint16_t x, uint16_t y) {
  const uint8_t a = x & 0xFF, b = x >> 8, c = y & 0xFF, d = y >> 8;
  const uint8_t ac = gf8b_mul(a, c), bd = gf8b_mul(b, d);
  const uint8_t lo = ac ^ gf8b_mul(0x20, bd);
  const uint8_t hi = gf8b_mul(a ^ b, c ^ d) ^ ac;
  return static_cast<uint16_t>(lo | (hi << 8));
}

inline uint16_t gf16_inv(uint16_t x) {
  if (!x) return 0;
  const uint8_t a = x & 0xFF, b = x >> 8;
  const uint8_t norm = gf8b_mul(a, a) ^ gf8b_mul(a, b) ^ gf8b_mul(0x20, gf8b_mul(b, b));
  const uint8_t ni = gf8b_tab().inv(norm);
  return static_cast<uint16_t>(gf8b_mul(a ^ b, ni) | (gf8b_mul(b, ni) << 8));
}

inline uint32_t gf32_mul(uint32_t x, uint32_t y) {
  const uint16_t a = x & 0xFFFF, b = x >> 16, c = y & 0xFFFF, d = y >> 16;
  const uint16_t ac = gf16_mul(a, c), bd = gf16_mul(b, d);
  const uint16_t lo = ac ^ gf16_mul(0x2000, bd);
  const uint16_t hi = gf16_mul(a ^ b, c ^ d) ^ ac;
  return static_cast<uint32_t>(lo) | (static_cast<uint32_t>(hi) << 16);
}

inline uint32_t gf32_inv(uint32_t x) {
  if (!x) return 0;
  const uint16_t a = x & 0xFFFF, b = x >> 16;
  const uint16_t norm = gf16_mul(a, a) ^ gf16_mul(a, b) ^ gf16_mul(0x2000, gf16_mul(b, b));
  const uint16_t ni = gf16_inv(norm);
  return static_cast<uint32_t>(gf16_mul(a ^ b, ni)) | (static_cast<uint32_t>(gf16_mul(b, ni)) << 16);
}

inline uint32_t gf_mul(int f, uint32_t a, uint32_t b) {
  switch (f) {
    case kGf8B: return gf8b_tab().mul(a & 0xFF, b & 0xFF);
    case kGf8D: return gf8d_tab().mul(a & 0xFF, b & 0xFF);
    case kGf16: return gf16_mul(a & 0xFFFF, b & 0xFFFF);
    case kGf32: return gf32_mul(a, b);
    default: return 0;
  }
}

inline uint32_t gf_inv(int f, uint32_t a) {
  switch (f) {
    case kGf8B: return gf8b_tab().inv(a & 0xFF);
    case kGf8D: return gf8d_tab().inv(a & 0xFF);
    case kGf16: return gf16_inv(a & 0xFFFF);
    case kGf32: return gf32_inv(a);
    default: return 0;
  }
}

// Multiplying a packed element by a fixed coefficient is linear over the
// byte subfield: output byte o = XOR_p M[o][p] * input byte p, products in
// the byte field (Gf8D for Gf8D, Gf8B otherwise). Fills M[0..E)[0..E).
//   Gf8 : M = [c]
//   Gf16: (a + b u)(c0 + c1 u) = (c0 a + 0x20 c1 b) + (c1 a + (c0 + c1) b) u
//   Gf32: the same identity one level up, each Gf16 product a 2x2 block.
inline void coeff_byte_matrix(int f, uint32_t c, uint8_t M[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) M[i][j] = 0;
  if (f == kGf8B || f == kGf8D) {
    M[0][0] = c & 0xFF;
    return;
  }
  auto m16 = [](uint16_t x, uint8_t out[2][2]) {
    const uint8_t x0 = x & 0xFF, x1 = x >> 8;
    out[0][0] = x0;
    out[0][1] = gf8b_mul(0x20, x1);
    out[1][0] = x1;
    out[1][1] = x0 ^ x1;
  };
  if (f == kGf16) {
    uint8_t b[2][2];
    m16(static_cast<uint16_t>(c), b);
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) M[i][j] = b[i][j];
    return;
  }
  const uint16_t c0 = c & 0xFFFF, c1 = c >> 16;
  const uint16_t blocks[2][2] = {{c0, gf16_mul(0x2000, c1)}, {c1, static_cast<uint16_t>(c0 ^ c1)}};
  for (int bi = 0; bi < 2; ++bi)
    for (int bj = 0; bj < 2; ++bj) {
      uint8_t b[2][2];
      m16(blocks[bi][bj], b);
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) M[2 * bi + i][2 * bj + j] = b[i][j];
    }
}

// Byte-subfield product used by the tables of field f.
inline uint8_t byte_mul(int f, uint8_t a, uint8_t b) {
  return f == kGf8D ? gf8d_tab().mul(a, b) : gf8b_tab().mul(a, b);
}

}  // namespace fgfc
