// gf_host.hpp -- host-side field arithmetic used to derive device tables and
// decode matrices. Product code (independent of the oracle under oracle/).
//
// Field definitions follow the reference crate:
//   Gf8B: GF(2)[x]/(x^8+x^4+x^3+x+1), generator 0x03     (src/field/gf8b.rs:57)
//   Gf8D: GF(2)[x]/(x^8+x^4+x^3+x^2+1), generator 0x02   (src/field/gf8d.rs:40)
//   Gf16: Gf8B[u]/(u^2+u+0x20), element a + b*u stored [a, b]  (src/field/gf16.rs:54-60)
//   Gf32: Gf16[v]/(v^2+v+0x2000), element a + b*v stored LE    (src/field/gf32.rs:36-42)
//   Gf64: Gf32[w]/(w^2+w+0x20000000), element a + b*w stored LE (src/field/gf64.rs:1-11)
//   Fp8/Fp16/Fp32/Fp64: the canonical Fan-Paar tower: the 2h-bit level is
//         h-bit[X]/(X^2 + alpha X + 1), alpha the h-bit level's top generator,
//         element lo + hi*X stored LE                            (src/field/fan_paar.rs:1-150)
// inv(0) = 0 and x/0 = 0 by convention (src/field/mod.rs:38-41).
#pragma once
#include <cstddef>
#include <cstdint>

namespace fgfc {

enum Field : int { kGf8B = 0, kGf8D = 1, kGf16 = 2, kGf32 = 3, kFp8 = 4, kFp16 = 5, kFp32 = 6, kGf64 = 7, kFp64 = 8 };

inline int field_bytes(int f) {
  switch (f) {
    case kGf8B:
    case kGf8D:
    case kFp8: return 1;
    case kGf16:
    case kFp16: return 2;
    case kGf32:
    case kFp32: return 4;
    case kGf64:
    case kFp64: return 8;
    default: return 0;
  }
}
inline const char* field_name(int f) {
  switch (f) {
    case kGf8B: return "GF(2^8)";
    case kGf8D: return "GF(2^8)/0x11D";
    case kGf16: return "GF(2^16)";
    case kGf32: return "GF(2^32)";
    case kFp8: return "Fan-Paar GF(2^8)";
    case kFp16: return "Fan-Paar GF(2^16)";
    case kFp32: return "Fan-Paar GF(2^32)";
    case kGf64: return "GF(2^64)";
    case kFp64: return "Fan-Paar GF(2^64)";
    default: return "?";
  }
}
inline uint64_t field_mask(int f) {
  const int E = field_bytes(f);
  return E >= 8 ? ~0ull : ((1ull << (8 * E)) - 1ull);
}

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

// Fan-Paar tower arithmetic over `bits`-bit values (bits a power of two).
// Products recurse by Karatsuba, z = (z0 + z2) + (z1 + alpha z2) X with
// z0 = a0 b0, z2 = a1 b1, z1 = (a0 + a1)(b0 + b1) + z0 + z2; multiplying by
// alpha (the level's top generator) is the linear recurrence
// alpha (a0 + a1 X) = a1 + (a0 + alpha' a1) X one level down; the inverse is
// the conjugate (a0 + alpha a1) - a1 X over the norm a0 (a0 + alpha a1) + a1^2.
inline uint64_t fp_low(unsigned bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1ull); }

inline uint64_t fp_mul_alpha(uint64_t v, unsigned bits) {
  if (bits == 1) return v & 1u;
  const unsigned h = bits / 2;
  const uint64_t a0 = v & fp_low(h), a1 = v >> h;
  return a1 | ((a0 ^ fp_mul_alpha(a1, h)) << h);
}

inline uint64_t fp_mul(uint64_t x, uint64_t y, unsigned bits) {
  if (bits == 1) return x & y & 1u;
  const unsigned h = bits / 2;
  const uint64_t m = fp_low(h);
  const uint64_t a0 = x & m, a1 = x >> h, b0 = y & m, b1 = y >> h;
  const uint64_t z0 = fp_mul(a0, b0, h), z2 = fp_mul(a1, b1, h);
  const uint64_t z1 = fp_mul(a0 ^ a1, b0 ^ b1, h) ^ z0 ^ z2;
  return (z0 ^ z2) | ((z1 ^ fp_mul_alpha(z2, h)) << h);
}

inline uint64_t fp_inv(uint64_t x, unsigned bits) {
  if (bits == 1) return x & 1u;
  const unsigned h = bits / 2;
  const uint64_t a0 = x & fp_low(h), a1 = x >> h;
  const uint64_t conj0 = a0 ^ fp_mul_alpha(a1, h);
  const uint64_t ni = fp_inv(fp_mul(a0, conj0, h) ^ fp_mul(a1, a1, h), h);
  return fp_mul(ni, conj0, h) | (fp_mul(ni, a1, h) << h);
}

inline unsigned fp_bits(int f) { return 8u * static_cast<unsigned>(field_bytes(f)); }

inline uint64_t gf64_mul(uint64_t x, uint64_t y) {
  const uint32_t a = static_cast<uint32_t>(x), b = static_cast<uint32_t>(x >> 32);
  const uint32_t c = static_cast<uint32_t>(y), d = static_cast<uint32_t>(y >> 32);
  const uint32_t ac = gf32_mul(a, c), bd = gf32_mul(b, d);
  const uint32_t lo = ac ^ gf32_mul(0x20000000u, bd);
  const uint32_t hi = gf32_mul(a ^ b, c ^ d) ^ ac;
  return static_cast<uint64_t>(lo) | (static_cast<uint64_t>(hi) << 32);
}

inline uint64_t gf64_inv(uint64_t x) {
  if (!x) return 0;
  const uint32_t a = static_cast<uint32_t>(x), b = static_cast<uint32_t>(x >> 32);
  const uint32_t norm = gf32_mul(a, a) ^ gf32_mul(a, b) ^ gf32_mul(0x20000000u, gf32_mul(b, b));
  const uint32_t ni = gf32_inv(norm);
  return static_cast<uint64_t>(gf32_mul(a ^ b, ni)) | (static_cast<uint64_t>(gf32_mul(b, ni)) << 32);
}

inline uint64_t gf_mul(int f, uint64_t a, uint64_t b) {
  switch (f) {
    case kGf8B: return gf8b_tab().mul(a & 0xFF, b & 0xFF);
    case kGf8D: return gf8d_tab().mul(a & 0xFF, b & 0xFF);
    case kGf16: return gf16_mul(a & 0xFFFF, b & 0xFFFF);
    case kGf32: return gf32_mul(static_cast<uint32_t>(a), static_cast<uint32_t>(b));
    case kFp8:
    case kFp16:
    case kFp32:
    case kFp64: return fp_mul(a & field_mask(f), b & field_mask(f), fp_bits(f));
    case kGf64: return gf64_mul(a, b);
    default: return 0;
  }
}

inline uint64_t gf_inv(int f, uint64_t a) {
  switch (f) {
    case kGf8B: return gf8b_tab().inv(a & 0xFF);
    case kGf8D: return gf8d_tab().inv(a & 0xFF);
    case kGf16: return gf16_inv(a & 0xFFFF);
    case kGf32: return gf32_inv(static_cast<uint32_t>(a));
    case kFp8:
    case kFp16:
    case kFp32:
    case kFp64: return fp_inv(a & field_mask(f), fp_bits(f));
    case kGf64: return gf64_inv(a);
    default: return 0;
  }
}

// Multiplying a packed element by a fixed coefficient c is linear over
// GF(2) in every field here. img[p][b] is c times the element whose only set
// bit is bit b of byte p (an E-byte value), so that for an input element x,
// byte o of c * x = XOR over the set bits (p, b) of x of byte o of img[p][b].
// Every table the kernels use (nibble and byte tables, GF(2) bit matrices)
// is derived from these images, for any field.
inline void coeff_images(int f, uint64_t c, uint64_t img[8][8]) {
  const int E = field_bytes(f);
  for (int p = 0; p < 8; ++p)
    for (int b = 0; b < 8; ++b)
      img[p][b] = p < E ? gf_mul(f, c & field_mask(f), 1ull << (8 * p + b)) : 0ull;
}

// Byte o of c * (x placed in input byte p), from the images.
inline uint8_t image_byte(const uint64_t img[8][8], int p, uint8_t x, int o) {
  uint64_t v = 0;
  for (int b = 0; b < 8; ++b)
    if ((x >> b) & 1u) v ^= img[p][b];
  return static_cast<uint8_t>(v >> (8 * o));
}

}  // namespace fgfc
