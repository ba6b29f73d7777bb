"""Coding and decode matrices for systematic codes [I_k ; C] through the C ABI
(`fgfc_cauchy_matrix`, `fgfc_decode_matrix`, `fgfc_decode_plan_create`).

The reference crate leaves these recipes to its callers (src/lib.rs:115-116);
its round-trip test solves for erased rows with scalar inverses under the
inv(0) = 0 convention (tests/ops.rs:897-950). Host computation in the library.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from ._lib import check, lib
from .ops import Plan, _fid


def cauchy_matrix(field, m: int, k: int, x0: int | None = None) -> list[list[int]]:
    """Row-major m x k parity matrix c[i][j] = inv(x_i + y_j), x_i = x0 + i (default k), y_j = j."""
    out = (C.c_uint32 * max(1, m * k))()
    check(lib().fgfc_cauchy_matrix(_fid(field), m, k, k if x0 is None else x0, out))
    return [[out[i * k + j] for j in range(k)] for i in range(m)]


def _args(parity: Sequence[Sequence[int]], survivors: Sequence[int], erased: Sequence[int]):
    m = len(parity)
    k = len(survivors)
    flat = (C.c_uint32 * max(1, m * k))(*[int(v) for row in parity for v in row])
    sv = (C.c_size_t * max(1, k))(*[int(s) for s in survivors])
    er = (C.c_size_t * max(1, len(erased)))(*[int(e) for e in erased])
    return flat, k, m, sv, er


def decode_matrix(field, parity: Sequence[Sequence[int]], survivors: Sequence[int],
                  erased: Sequence[int]) -> list[int]:
    """Decode rows, term-major (out[t * len(erased) + e]): the Plan::matrix(k, len(erased)) layout."""
    flat, k, m, sv, er = _args(parity, survivors, erased)
    out = (C.c_uint32 * max(1, k * len(erased)))()
    check(lib().fgfc_decode_matrix(_fid(field), flat, k, m, sv, er, len(erased), out))
    return list(out[:k * len(erased)])


def decode_plan(field, parity: Sequence[Sequence[int]], survivors: Sequence[int], erased: Sequence[int]) -> Plan:
    """The decode rows as a device plan of dimensions (k, len(erased))."""
    flat, k, m, sv, er = _args(parity, survivors, erased)
    h = C.c_void_p()
    check(lib().fgfc_decode_plan_create(_fid(field), flat, k, m, sv, er, len(erased), C.byref(h)))
    return Plan._adopt(field, h, k, len(erased))
