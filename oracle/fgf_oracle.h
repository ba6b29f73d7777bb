/*
 * fgf_oracle.h -- CPU oracle for the packed-vector ops hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a scalar C restatement of the reference
 * library's field arithmetic and elementwise op semantics, used to check the
 * CUDA path. Only the test suite, the smoke check and the CPU-baseline leg of
 * the benchmark may load it; the product library never links or calls it.
 *
 * Parity pin: the restatement is checked against every known-answer product,
 * doctest vector and table self-test in the reference's own test suite
 * (tests/algebra.rs, src/lib.rs, README.md, src/field/*.rs doctests,
 * src/kernel/tables.rs tests); see tests/test_oracle_pins.py.
 *
 * Field ids: 0 = Gf8B (0x11B), 1 = Gf8D (0x11D), 2 = Gf16 (tower over Gf8B),
 * 3 = Gf32 (tower over Gf16), 4 / 5 / 6 = canonical Fan-Paar GF(2^8) /
 * GF(2^16) / GF(2^32), 7 = Gf64 (tower over Gf32), 8 = Fan-Paar GF(2^64).
 * Scalars are uint32_t (uint64_t in the *64 functions), op coefficients
 * uint64_t; buffers
 * hold packed little-endian elements exactly as the reference's `ops` does.
 *
 * Coefficient matrices for the many-to-many ops are passed term-major:
 * coeffs[t * nrows + j] multiplies source t into row j, which is the layout
 * of the reference's `Plan::matrix(sources, rows, ..)` (src/ops.rs:712-718).
 */
#ifndef FGF_ORACLE_H
#define FGF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_GF8B = 0, ORC_GF8D = 1, ORC_GF16 = 2, ORC_GF32 = 3, ORC_FP8 = 4, ORC_FP16 = 5, ORC_FP32 = 6,
       ORC_GF64 = 7, ORC_FP64 = 8 };

int orc_bytes(int field);

/* Scalar field arithmetic. */
uint32_t orc_mul(int field, uint32_t a, uint32_t b);
uint32_t orc_mul_xtime(int field, uint32_t a, uint32_t b); /* Gf8 shift/XOR form */
uint32_t orc_inv(int field, uint32_t a);                   /* inv(0) == 0 */
uint32_t orc_inv_xtime(int field, uint32_t a);             /* Gf8 Fermat form */
uint32_t orc_div(int field, uint32_t a, uint32_t b);       /* x / 0 == 0 */
uint32_t orc_pow(int field, uint32_t a, uint64_t e);
uint32_t orc_square(int field, uint32_t a);
/* The same for every field, 8-byte ones included (values as uint64_t). */
uint64_t orc_mul64(int field, uint64_t a, uint64_t b);
uint64_t orc_inv64(int field, uint64_t a);
uint64_t orc_pow64(int field, uint64_t a, uint64_t e);

/* The reference tests' deterministic byte stream (tests/ops.rs:17-27). */
void orc_noise(uint8_t *out, size_t len, uint64_t seed);

/* Elementwise op semantics (src/kernel/scalar.rs, src/ops.rs). */
void orc_xor(uint8_t *dst, const uint8_t *src, size_t len);
void orc_mul_add(int field, uint8_t *dst, uint64_t coeff, const uint8_t *src, size_t len);
void orc_mul_into(int field, uint8_t *dst, uint64_t coeff, const uint8_t *src, size_t len);
void orc_mul_assign(int field, uint8_t *dst, uint64_t coeff, size_t len);
void orc_mul_elementwise(int field, uint8_t *dst, const uint8_t *a, const uint8_t *b, size_t len);
void orc_mul_add_scatter(int field, uint8_t *rows, size_t row_len, const uint64_t *coeffs,
                         size_t nrows, const uint8_t *src);
void orc_mul_add_gather(int field, uint8_t *dst, size_t len, const uint64_t *coeffs,
                        const uint8_t *const *srcs, size_t nsrcs);
void orc_dot_product(int field, uint8_t *dst, size_t len, const uint64_t *coeffs,
                     const uint8_t *const *srcs, size_t nsrcs);
void orc_mul_add_matrix(int field, uint8_t *rows, size_t row_len, size_t nrows,
                        const uint64_t *coeffs, const uint8_t *const *srcs, size_t nsrcs);
void orc_dot_product_matrix(int field, uint8_t *rows, size_t row_len, size_t nrows,
                            const uint64_t *coeffs, const uint8_t *const *srcs, size_t nsrcs);
void orc_mul_add_matrix_scattered(int field, uint8_t *dst, size_t row_len,
                                  const size_t *row_starts, size_t nrows,
                                  const uint64_t *coeffs, const uint8_t *const *srcs,
                                  size_t nsrcs);

/* Reed-Solomon recipes built on the field arithmetic (caller-side in the
 * reference: src/lib.rs:115-116; Cramer example tests/ops.rs:897-950). */
/* c[i * k + j] = inv(x_i + y_j), x_i = x0 + i, y_j = j, for i < m, j < k. */
void orc_cauchy(int field, uint32_t *c, size_t m, size_t k, uint32_t x0);
/* In-place Gauss-Jordan inverse of an n x n row-major matrix; 0 on success,
 * -1 if singular. Uses inv(0) == 0 only on nonzero pivots. */
int orc_invert(int field, uint32_t *a, size_t n);
/* Decode rows for a systematic code with generator [I_k ; C] (C is m x k).
 * survivors: k codeword indices in [0, k+m); erased: r indices.
 * out[j * k + t] = coefficient of survivor t in erased row j.
 * Returns 0, or -1 if the survivor submatrix is singular. */
int orc_decode_matrix(int field, const uint32_t *c, size_t k, size_t m,
                      const size_t *survivors, const size_t *erased, size_t r, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif
