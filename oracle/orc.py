"""ctypes wrapper over liborc.so, the CPU oracle (test infrastructure only).

Functions take and return numpy uint8 arrays; coefficient matrices are
term-major (coeffs[t * nrows + j]), the layout of the reference's
Plan::matrix(sources, rows, ..) (src/ops.rs:712-718).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

GF8B, GF8D, GF16, GF32 = 0, 1, 2, 3
FP8, FP16, FP32 = 4, 5, 6  # canonical Fan-Paar towers (src/field/fan_paar.rs)
GF64, FP64 = 7, 8  # GF(2^64) over GF(2^32) (src/field/gf64.rs), Fan-Paar GF(2^64)

_L: C.CDLL | None = None


def L() -> C.CDLL:
    global _L
    if _L is None:
        path = _build.LIB
        if not path.exists():
            _build.build()
        _L = C.CDLL(str(path))
        u32, sz, p = C.c_uint32, C.c_size_t, C.c_void_p
        for name in ("orc_mul", "orc_mul_xtime", "orc_div"):
            getattr(_L, name).restype = u32
            getattr(_L, name).argtypes = [C.c_int, u32, u32]
        for name in ("orc_inv", "orc_inv_xtime", "orc_square"):
            getattr(_L, name).restype = u32
            getattr(_L, name).argtypes = [C.c_int, u32]
        _L.orc_pow.restype = u32
        _L.orc_pow.argtypes = [C.c_int, u32, C.c_uint64]
        u64 = C.c_uint64
        _L.orc_mul64.restype = u64
        _L.orc_mul64.argtypes = [C.c_int, u64, u64]
        _L.orc_inv64.restype = u64
        _L.orc_inv64.argtypes = [C.c_int, u64]
        _L.orc_pow64.restype = u64
        _L.orc_pow64.argtypes = [C.c_int, u64, u64]
        _L.orc_noise.argtypes = [p, sz, C.c_uint64]
        _L.orc_invert.restype = C.c_int
        _L.orc_decode_matrix.restype = C.c_int
    return _L


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _u32(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.uint64).astype(np.uint32))


def _u64(v) -> np.ndarray:
    # Python ints are converted one by one: np.asarray of a list that mixes
    # values below and at or above 2^63 would go through float64 and round.
    if isinstance(v, np.ndarray):
        return np.ascontiguousarray(v.reshape(-1).astype(np.uint64))
    return np.ascontiguousarray(np.array([int(x) & 0xFFFFFFFFFFFFFFFF for x in v], dtype=np.uint64))


def _ptrs(srcs) -> C.Array:
    return (C.c_void_p * max(1, len(srcs)))(*[s.ctypes.data for s in srcs])


def mul(f, a, b):
    return L().orc_mul(f, a, b)


def mul_xtime(f, a, b):
    return L().orc_mul_xtime(f, a, b)


def inv(f, a):
    return L().orc_inv(f, a)


def inv_xtime(f, a):
    return L().orc_inv_xtime(f, a)


def div(f, a, b):
    return L().orc_div(f, a, b)


def pow_(f, a, e):
    return L().orc_pow(f, a, e)


def mul64(f, a, b):
    """Product in any field, 8-byte ones included."""
    return L().orc_mul64(f, a, b)


def inv64(f, a):
    return L().orc_inv64(f, a)


def pow64(f, a, e):
    return L().orc_pow64(f, a, e)


def noise(n: int, seed: int) -> np.ndarray:
    """The reference tests' LCG byte stream (tests/ops.rs:17-27)."""
    out = np.empty(n, dtype=np.uint8)
    if n:
        L().orc_noise(_p(out), n, seed & 0xFFFFFFFFFFFFFFFF)
    return out


def mul_add(f, dst: np.ndarray, c: int, src: np.ndarray) -> None:
    L().orc_mul_add(f, _p(dst), C.c_uint64(c), _p(src), C.c_size_t(len(dst)))


def mul_into(f, dst, c, src) -> None:
    L().orc_mul_into(f, _p(dst), C.c_uint64(c), _p(src), C.c_size_t(len(dst)))


def mul_assign(f, dst, c) -> None:
    L().orc_mul_assign(f, _p(dst), C.c_uint64(c), C.c_size_t(len(dst)))


def mul_elementwise(f, dst, a, b) -> None:
    L().orc_mul_elementwise(f, _p(dst), _p(a), _p(b), C.c_size_t(len(dst)))


def mul_add_scatter(f, rows, row_len, coeffs, src) -> None:
    c = _u64(coeffs)
    L().orc_mul_add_scatter(f, _p(rows), C.c_size_t(row_len), _p(c), C.c_size_t(len(c)), _p(src))


def mul_add_gather(f, dst, coeffs, srcs) -> None:
    c = _u64(coeffs)
    L().orc_mul_add_gather(f, _p(dst), C.c_size_t(len(dst)), _p(c), _ptrs(srcs), C.c_size_t(len(srcs)))


def dot_product(f, dst, coeffs, srcs) -> None:
    c = _u64(coeffs)
    L().orc_dot_product(f, _p(dst), C.c_size_t(len(dst)), _p(c), _ptrs(srcs), C.c_size_t(len(srcs)))


def mul_add_matrix(f, rows, row_len, nrows, coeffs, srcs) -> None:
    c = _u64(coeffs)
    L().orc_mul_add_matrix(f, _p(rows), C.c_size_t(row_len), C.c_size_t(nrows), _p(c), _ptrs(srcs),
                           C.c_size_t(len(srcs)))


def dot_product_matrix(f, rows, row_len, nrows, coeffs, srcs) -> None:
    c = _u64(coeffs)
    L().orc_dot_product_matrix(f, _p(rows), C.c_size_t(row_len), C.c_size_t(nrows), _p(c), _ptrs(srcs),
                               C.c_size_t(len(srcs)))


def mul_add_matrix_scattered(f, dst, row_len, row_starts, coeffs, srcs) -> None:
    c = _u64(coeffs)
    st = (C.c_size_t * max(1, len(row_starts)))(*row_starts)
    L().orc_mul_add_matrix_scattered(f, _p(dst), C.c_size_t(row_len), st, C.c_size_t(len(row_starts)),
                                     _p(c), _ptrs(srcs), C.c_size_t(len(srcs)))


def cauchy(f, m, k, x0=None) -> np.ndarray:
    out = np.zeros(m * k, dtype=np.uint32)
    L().orc_cauchy(f, _p(out), C.c_size_t(m), C.c_size_t(k), C.c_uint32(k if x0 is None else x0))
    return out.reshape(m, k)


def decode_matrix(f, c: np.ndarray, survivors, erased) -> np.ndarray:
    m, k = c.shape
    cc = _u32(c.reshape(-1))
    sv = (C.c_size_t * k)(*survivors)
    er = (C.c_size_t * max(1, len(erased)))(*erased)
    out = np.zeros(len(erased) * k, dtype=np.uint32)
    rc = L().orc_decode_matrix(f, _p(cc), C.c_size_t(k), C.c_size_t(m), sv, er, C.c_size_t(len(erased)),
                               _p(out))
    if rc != 0:
        raise ValueError("singular survivor submatrix")
    return out.reshape(len(erased), k)
