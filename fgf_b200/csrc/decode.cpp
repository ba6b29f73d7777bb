// decode.cpp -- coding and decode matrices for systematic codes [I_k ; C].
//
// The reference leaves coding-matrix construction and decoding to its
// callers (src/lib.rs:115-116); its own round-trip test inverts a survivor
// submatrix by Cramer's rule with scalar field inverses (tests/ops.rs:897-950),
// where inv(0) = 0 by convention (src/field/mod.rs:38-41,
// src/field/flat8.rs:377-399). This file gives a caller of the C ABI the same
// recipes natively, so a reconstruct can be requested by erasure pattern:
//   * Cauchy parity matrices c[i][j] = inv(x_i + y_j), x_i = x0 + i, y_j = j;
//   * decode rows: for k surviving shard indices (0..k-1 data, k..k+m-1
//     parity) the k x k submatrix of [I_k ; C] is inverted by Gauss-Jordan
//     elimination over the field, and erased shard e is
//     sum_t D[e][t] * survivor_t with D[e] = G[e] * inv(S).
// Field arithmetic is gf_host.hpp's (product code, independent of the oracle).
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.hpp"

namespace fgfc {

namespace {

// Row-major n x n inverse over `field`; false if singular.
bool invert(int field, std::vector<uint32_t>& a, size_t n, std::vector<uint32_t>& inv) {
  inv.assign(n * n, 0);
  for (size_t i = 0; i < n; ++i) inv[i * n + i] = 1;
  for (size_t col = 0; col < n; ++col) {
    size_t piv = col;
    while (piv < n && a[piv * n + col] == 0) ++piv;
    if (piv == n) return false;
    if (piv != col)
      for (size_t x = 0; x < n; ++x) {
        std::swap(a[piv * n + x], a[col * n + x]);
        std::swap(inv[piv * n + x], inv[col * n + x]);
      }
    const uint32_t pinv = gf_inv(field, a[col * n + col]);
    for (size_t x = 0; x < n; ++x) {
      a[col * n + x] = gf_mul(field, a[col * n + x], pinv);
      inv[col * n + x] = gf_mul(field, inv[col * n + x], pinv);
    }
    for (size_t r = 0; r < n; ++r) {
      const uint32_t f = a[r * n + col];
      if (r == col || f == 0) continue;
      for (size_t x = 0; x < n; ++x) {
        a[r * n + x] ^= gf_mul(field, f, a[col * n + x]);
        inv[r * n + x] ^= gf_mul(field, f, inv[col * n + x]);
      }
    }
  }
  return true;
}

// Row `r` of the generator [I_k ; C] (C row-major m x k).
inline uint32_t gen_at(const uint32_t* parity, size_t k, size_t r, size_t col) {
  return r < k ? (r == col ? 1u : 0u) : parity[(r - k) * k + col];
}

}  // namespace

// Decode rows, term-major (out[t * nerased + e]); returns 0 or an fgfc_status
// with the error text set.
fgfc_status decode_matrix(int field, const uint32_t* parity, size_t k, size_t m, const size_t* survivors,
                          const size_t* erased, size_t nerased, uint32_t* out) {
  const char* name = "decode_matrix";
  if (field_bytes(field) == 0) return set_error(FGFC_ERR_ARG, "decode_matrix: unknown field");
  if (field_bytes(field) > 4)
    return set_error(FGFC_ERR_ARG, "decode_matrix: 8-byte fields need 64-bit coefficients, which these 32-bit "
                                   "arrays cannot hold");
  if (!k || (m && !parity) || !survivors || (nerased && (!erased || !out)))
    return set_error(FGFC_ERR_ARG, "decode_matrix: null argument");
  const uint32_t mask = field_mask(field);
  std::vector<char> seen(k + m, 0);
  for (size_t t = 0; t < k; ++t) {
    if (survivors[t] >= k + m || seen[survivors[t]]) {
      char msg[160];
      snprintf(msg, sizeof msg, "%s: survivor %zu is out of range or repeated", name, survivors[t]);
      return set_error(FGFC_ERR_ARG, msg);
    }
    seen[survivors[t]] = 1;
  }
  for (size_t e = 0; e < nerased; ++e)
    if (erased[e] >= k + m) {
      char msg[160];
      snprintf(msg, sizeof msg, "%s: erased shard %zu is out of range", name, erased[e]);
      return set_error(FGFC_ERR_ARG, msg);
    }
  std::vector<uint32_t> sub(k * k), inv;
  for (size_t t = 0; t < k; ++t)
    for (size_t c = 0; c < k; ++c) sub[t * k + c] = gen_at(parity, k, survivors[t], c) & mask;
  if (!invert(field, sub, k, inv)) return set_error(FGFC_ERR_ARG, "decode_matrix: the survivor submatrix is singular");
  // shard e = G[e] . data, data = inv . survivors  =>  D[e][t] = sum_q G[e][q] inv[q][t]
  for (size_t e = 0; e < nerased; ++e)
    for (size_t t = 0; t < k; ++t) {
      uint32_t acc = 0;
      for (size_t q = 0; q < k; ++q) acc ^= gf_mul(field, gen_at(parity, k, erased[e], q) & mask, inv[q * k + t]);
      out[t * nerased + e] = acc;
    }
  return clear_error();
}

}  // namespace fgfc

using namespace fgfc;

extern "C" {

fgfc_status fgfc_cauchy_matrix(fgfc_field field, size_t m, size_t k, uint32_t x0, uint32_t* out) {
  if (field_bytes(field) == 0 || (m * k && !out)) return set_error(FGFC_ERR_ARG, "cauchy_matrix: invalid argument");
  if (field_bytes(field) > 4)
    return set_error(FGFC_ERR_ARG, "cauchy_matrix: 8-byte fields need 64-bit coefficients, which these 32-bit "
                                   "arrays cannot hold");
  for (size_t i = 0; i < m; ++i)
    for (size_t j = 0; j < k; ++j) {
      const uint32_t x = static_cast<uint32_t>(x0 + i), y = static_cast<uint32_t>(j);
      if (((x ^ y) & field_mask(field)) == 0 || (x & ~field_mask(field)) || (y & ~field_mask(field)))
        return set_error(FGFC_ERR_ARG, "cauchy_matrix: x_i + y_j must be nonzero field elements");
      out[i * k + j] = gf_inv(field, x ^ y);
    }
  return clear_error();
}

fgfc_status fgfc_decode_matrix(fgfc_field field, const uint32_t* parity, size_t k, size_t m, const size_t* survivors,
                               const size_t* erased, size_t nerased, uint32_t* out) {
  return decode_matrix(field, parity, k, m, survivors, erased, nerased, out);
}

fgfc_status fgfc_decode_plan_create(fgfc_field field, const uint32_t* parity, size_t k, size_t m,
                                    const size_t* survivors, const size_t* erased, size_t nerased, fgfc_plan** out) {
  if (!out) return set_error(FGFC_ERR_ARG, "decode_plan_create: null argument");
  std::vector<uint32_t> d(k * nerased + 1);
  fgfc_status st = decode_matrix(field, parity, k, m, survivors, erased, nerased, d.data());
  if (st != FGFC_OK) return st;
  return fgfc_plan_create(field, k, nerased, d.data(), out);
}

}  // extern "C"
