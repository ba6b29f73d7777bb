"""The `fgf::ops` surface over device buffers.

Every function mirrors the reference function of the same name in
src/ops.rs: same argument order and meaning, the field passed first where
the reference takes a type parameter (`ops::mul_add::<Gf8D>(dst, c, src)`
becomes `ops.mul_add(Gf8D, dst, c, src)`). Buffers are device memory: CUDA
uint8 torch tensors (any contiguous view) or `(device_pointer, nbytes)`
pairs. Calls are asynchronous on `stream` (default: torch's current
stream). A call the reference would reject with a panic raises `FgfError`
carrying the reference's message.

All computation happens in libfgfcuda.so; this module only marshals
arguments through the C ABI (include/fgf_cuda.h).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Sequence

from ._lib import FgfError, Slice, Term, check, lib
from .fields import FIELDS, Gf8B, Gf8D, Gf16, Gf32  # noqa: F401  (re-exported markers)

__all__ = [
    "FgfError", "Coeff", "CoeffRef", "Plan",
    "add_assign", "sub_assign", "mul_add", "mul_add_with", "mul_into", "mul_into_with",
    "mul_assign", "mul_assign_with", "mul_add_scatter", "mul_add_scatter_with",
    "mul_add_gather", "mul_add_gather_with", "dot_product", "dot_product_with",
    "mul_add_matrix", "mul_add_matrix_with", "dot_product_matrix", "dot_product_matrix_with",
    "mul_add_matrix_scattered", "mul_add_matrix_scattered_with", "mul_elementwise",
    "pack", "unpack", "pack_to_vec",
]


# ---------------------------------------------------------------- buffers / streams

def _buf(x) -> tuple[int, int]:
    """(device pointer, byte length) of a device buffer."""
    if isinstance(x, tuple):
        return int(x[0]), int(x[1])
    try:
        on_device = x.is_cuda
    except AttributeError:
        raise TypeError(f"fgf_b200.ops: unsupported buffer type {type(x).__name__}") from None
    if not on_device:
        raise TypeError("fgf_b200.ops: buffers must be device (CUDA) memory")
    if not x.is_contiguous():
        raise TypeError("fgf_b200.ops: buffers must be contiguous")
    return x.data_ptr(), x.nbytes


def _stream(stream) -> int:
    if stream is None:
        try:
            import torch

            if torch.cuda.is_available() and torch.cuda.is_initialized():
                return int(torch.cuda.current_stream().cuda_stream)
        except ImportError:
            pass
        return 0
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    return int(stream)


def _u32s(values: Iterable[int]):
    vals = [int(v) & 0xFFFFFFFF for v in values]
    return (C.c_uint32 * max(1, len(vals)))(*vals), len(vals)


def _u64s(values: Iterable[int]):
    vals = [int(v) & 0xFFFFFFFFFFFFFFFF for v in values]
    return (C.c_uint64 * max(1, len(vals)))(*vals), len(vals)


def _wide(field) -> bool:
    """8-byte fields: their coefficients are 64-bit, so the raw forms below
    prepare a plan and run the prepared form (the C ABI's raw entry points
    take 32-bit coefficients)."""
    return FIELDS[_fid(field)].BYTES == 8


_SLICE_WORDS: dict = {}


def _slices(srcs: Sequence):
    """fgfc_slice array of the sources: built as one flat array of (pointer,
    length) words (one ctypes object instead of one per source) and viewed
    as the struct array, which keeps the words alive."""
    flat = []
    for s in srcs:
        flat.extend(_buf(s))
    n = len(flat) // 2
    typ = _SLICE_WORDS.get(n)
    if typ is None:
        typ = _SLICE_WORDS[n] = C.c_uint64 * max(2, 2 * n)
    return C.cast(typ(*flat), C.POINTER(Slice)), n


def _terms(terms: Sequence) -> tuple[C.Array, int, list]:
    keep = []
    out = []
    for coeffs, src in terms:
        carr, n = _u32s(coeffs)
        keep.append(carr)
        p, ln = _buf(src)
        out.append(Term(C.cast(carr, C.POINTER(C.c_uint32)), n, p, ln))
    arr = (Term * max(1, len(out)))(*out)
    return arr, len(out), keep


def _fid(field) -> int:
    return field.ID if hasattr(field, "ID") else int(field)


# ---------------------------------------------------------------- Plan / Coeff

class Plan:
    """`ops::Plan<F>` (src/ops.rs:158-276): coefficients prepared once and
    uploaded to the device; `get`/`get_at`/`row` borrow entries."""

    def __init__(self, field, coeffs: Sequence[int], _rows: int | None = None, _cols: int | None = None):
        self.field = FIELDS[_fid(field)]
        vals = [int(v) for v in coeffs]
        rows = 1 if _rows is None else _rows
        cols = len(vals) if _cols is None else _cols
        arr, _ = _u64s(vals)
        h = C.c_void_p()
        check(lib().fgfc_plan_create_u64(self.field.ID, rows, cols, arr, C.byref(h)))
        self._h = h
        self._values = [v & ((1 << (8 * self.field.BYTES)) - 1) for v in vals]
        self._rows, self._cols = rows, cols

    @classmethod
    def new(cls, field, coeffs: Sequence[int]) -> "Plan":
        return cls(field, coeffs)

    @classmethod
    def _adopt(cls, field, handle: C.c_void_p, rows: int, cols: int) -> "Plan":
        """Wrap a plan the library created (e.g. fgfc_decode_plan_create)."""
        self = cls.__new__(cls)
        self.field = FIELDS[_fid(field)]
        self._h = handle
        vals = (C.c_uint64 * max(1, rows * cols))()
        check(lib().fgfc_plan_values_u64(handle, vals))
        self._values = list(vals[:rows * cols])
        self._rows, self._cols = rows, cols
        return self

    @classmethod
    def matrix(cls, field, rows: int, cols: int, coeffs: Sequence[int]) -> "Plan":
        if rows * cols != len(coeffs):
            # ops.rs:199-207 (the C ABI reports the same condition; checked
            # here first so the message carries the caller's counts)
            raise FgfError(4, f"Plan::matrix: {len(coeffs)} coefficients for {rows}x{cols} matrix")
        return cls(field, coeffs, rows, cols)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value:
            try:
                lib().fgfc_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def __len__(self) -> int:
        return len(self._values)

    def len(self) -> int:
        return len(self._values)

    def is_empty(self) -> bool:
        return not self._values

    def dimensions(self) -> tuple[int, int]:
        return (self._rows, self._cols)

    def values(self) -> list[int]:
        return list(self._values)

    def get(self, index: int) -> "CoeffRef | None":
        return CoeffRef(self, index) if 0 <= index < len(self._values) else None

    def get_at(self, row: int, col: int) -> "CoeffRef | None":
        if 0 <= row < self._rows and 0 <= col < self._cols:
            return self.get(row * self._cols + col)
        return None

    def row(self, row: int) -> "list[CoeffRef] | None":
        start = row * self._cols
        if row < 0 or start + self._cols > len(self._values):
            return None
        return [CoeffRef(self, start + i) for i in range(self._cols)]

    def coeffs(self) -> "list[CoeffRef]":
        return [CoeffRef(self, i) for i in range(len(self._values))]

    def __repr__(self) -> str:
        return f"Plan {{ dimensions: {self.dimensions()}, len: {len(self)}, .. }}"


class Coeff(Plan):
    """`ops::Coeff<F>` (src/ops.rs:44-73): a single prepared coefficient."""

    def __init__(self, field, coeff: int):
        super().__init__(field, [coeff], 1, 1)

    def value(self) -> int:
        return self._values[0]

    def __repr__(self) -> str:
        return f"Coeff({self.value():#x})"


class CoeffRef:
    """`ops::CoeffRef` (src/ops.rs:121-156): a borrowed plan entry."""

    def __init__(self, plan: Plan, index: int):
        self.plan = plan
        self.index = index
        self.field = plan.field

    def value(self) -> int:
        return self.plan._values[self.index]


def _coeff_handle(coeff):
    """A 1-entry prepared coefficient handle, or None with the raw value."""
    if isinstance(coeff, Coeff):
        return coeff.field, coeff.handle, coeff.value()
    if isinstance(coeff, CoeffRef):
        if len(coeff.plan) == 1:
            return coeff.field, coeff.plan.handle, coeff.value()
        return coeff.field, None, coeff.value()
    raise TypeError("expected Coeff or CoeffRef")


# ---------------------------------------------------------------- single-row ops

def add_assign(field, dst, src, stream=None) -> None:
    """`dst ^= src` (src/ops.rs:323-326)."""
    d, dn = _buf(dst)
    s, sn = _buf(src)
    check(lib().fgfc_add_assign(_fid(field), d, dn, s, sn, _stream(stream)))


def sub_assign(field, dst, src, stream=None) -> None:
    """Identical to add_assign in characteristic two (src/ops.rs:333-335)."""
    add_assign(field, dst, src, stream)


def mul_add(field, dst, coeff: int, src, stream=None) -> None:
    """`dst ^= coeff * src` (src/ops.rs:342-352)."""
    if _wide(field):
        return mul_add_with(dst, Coeff(field, coeff), src, stream)
    d, dn = _buf(dst)
    s, sn = _buf(src)
    check(lib().fgfc_mul_add(_fid(field), d, dn, int(coeff) & 0xFFFFFFFF, s, sn, _stream(stream)))


def mul_add_with(dst, coeff, src, stream=None) -> None:
    """`dst ^= coeff * src` with a prepared coefficient (src/ops.rs:359-374)."""
    f, h, v = _coeff_handle(coeff)
    if h is None:
        return mul_add(f, dst, v, src, stream)
    d, dn = _buf(dst)
    s, sn = _buf(src)
    check(lib().fgfc_mul_add_with(d, dn, h, s, sn, _stream(stream)))


def mul_into(field, dst, coeff: int, src, stream=None) -> None:
    """`dst = coeff * src` (src/ops.rs:381-392)."""
    if _wide(field):
        return mul_into_with(dst, Coeff(field, coeff), src, stream)
    d, dn = _buf(dst)
    s, sn = _buf(src)
    check(lib().fgfc_mul_into(_fid(field), d, dn, int(coeff) & 0xFFFFFFFF, s, sn, _stream(stream)))


def mul_into_with(dst, coeff, src, stream=None) -> None:
    """src/ops.rs:399-415."""
    f, h, v = _coeff_handle(coeff)
    if h is None:
        return mul_into(f, dst, v, src, stream)
    d, dn = _buf(dst)
    s, sn = _buf(src)
    check(lib().fgfc_mul_into_with(d, dn, h, s, sn, _stream(stream)))


def mul_assign(field, dst, coeff: int, stream=None) -> None:
    """`dst *= coeff` in place (src/ops.rs:422-432)."""
    if _wide(field):
        return mul_assign_with(dst, Coeff(field, coeff), stream)
    d, dn = _buf(dst)
    check(lib().fgfc_mul_assign(_fid(field), d, dn, int(coeff) & 0xFFFFFFFF, _stream(stream)))


def mul_assign_with(dst, coeff, stream=None) -> None:
    """src/ops.rs:439-450."""
    f, h, v = _coeff_handle(coeff)
    if h is None:
        return mul_assign(f, dst, v, stream)
    d, dn = _buf(dst)
    check(lib().fgfc_mul_assign_with(d, dn, h, _stream(stream)))


def mul_elementwise(field, dst, a, b, stream=None) -> None:
    """`dst[i] = a[i] * b[i]` (src/ops.rs:953-957)."""
    d, dn = _buf(dst)
    pa, na = _buf(a)
    pb, nb = _buf(b)
    check(lib().fgfc_mul_elementwise(_fid(field), d, dn, pa, na, pb, nb, _stream(stream)))


# ---------------------------------------------------------------- scatter / gather / dot

def mul_add_scatter(field, rows, row_len: int, coeffs: Sequence[int], src, stream=None) -> None:
    """`rows[j] ^= coeffs[j] * src` (src/ops.rs:461-482)."""
    if _wide(field) and len(coeffs):
        return mul_add_scatter_with(rows, row_len, Plan.new(field, coeffs), src, stream)
    r, rn = _buf(rows)
    s, sn = _buf(src)
    arr, n = _u32s(coeffs)
    check(lib().fgfc_mul_add_scatter(_fid(field), r, rn, row_len, arr, n, s, sn, _stream(stream)))


def mul_add_scatter_with(rows, row_len: int, plan: Plan, src, stream=None) -> None:
    """src/ops.rs:493-520."""
    r, rn = _buf(rows)
    s, sn = _buf(src)
    check(lib().fgfc_mul_add_scatter_with(r, rn, row_len, plan.handle, s, sn, _stream(stream)))


def mul_add_gather(field, dst, coeffs: Sequence[int], srcs: Sequence, stream=None) -> None:
    """`dst ^= sum coeffs[i] * srcs[i]` (src/ops.rs:533-555)."""
    if _wide(field) and len(coeffs) and len(coeffs) == len(srcs):
        return mul_add_gather_with(dst, Plan.new(field, coeffs), srcs, stream)
    d, dn = _buf(dst)
    arr, n = _u32s(coeffs)
    sl, ns = _slices(srcs)
    check(lib().fgfc_mul_add_gather(_fid(field), d, dn, arr, n, sl, ns, _stream(stream)))


def mul_add_gather_with(dst, plan: Plan, srcs: Sequence, stream=None) -> None:
    """src/ops.rs:563-585."""
    d, dn = _buf(dst)
    sl, ns = _slices(srcs)
    check(lib().fgfc_mul_add_gather_with(d, dn, plan.handle, sl, ns, _stream(stream)))


def dot_product(field, dst, coeffs: Sequence[int], srcs: Sequence, stream=None) -> None:
    """`dst = sum coeffs[i] * srcs[i]` (src/ops.rs:597-624)."""
    if _wide(field) and len(coeffs) and len(coeffs) == len(srcs):
        return dot_product_with(dst, Plan.new(field, coeffs), srcs, stream)
    d, dn = _buf(dst)
    arr, n = _u32s(coeffs)
    sl, ns = _slices(srcs)
    check(lib().fgfc_dot_product(_fid(field), d, dn, arr, n, sl, ns, _stream(stream)))


def dot_product_with(dst, plan: Plan, srcs: Sequence, stream=None) -> None:
    """src/ops.rs:632-660."""
    d, dn = _buf(dst)
    sl, ns = _slices(srcs)
    check(lib().fgfc_dot_product_with(d, dn, plan.handle, sl, ns, _stream(stream)))


# ---------------------------------------------------------------- matrices

def mul_add_matrix(field, rows, row_len: int, nrows: int, terms: Sequence, stream=None) -> None:
    """`rows[j] ^= sum_t coeffs_t[j] * src_t` over `(coeffs, src)` terms (src/ops.rs:675-708)."""
    if _wide(field) and terms and all(len(c) == nrows for c, _ in terms):
        plan = Plan.matrix(field, len(terms), nrows, [int(v) for c, _ in terms for v in c])
        return mul_add_matrix_with(rows, row_len, nrows, plan, [src for _, src in terms], stream)
    r, rn = _buf(rows)
    arr, n, _keep = _terms(terms)
    check(lib().fgfc_mul_add_matrix(_fid(field), r, rn, row_len, nrows, arr, n, _stream(stream)))


def mul_add_matrix_with(rows, row_len: int, nrows: int, plan: Plan, srcs: Sequence, stream=None) -> None:
    """src/ops.rs:720-760; plan dimensions are (len(srcs), nrows)."""
    r, rn = _buf(rows)
    sl, ns = _slices(srcs)
    check(lib().fgfc_mul_add_matrix_with(r, rn, row_len, nrows, plan.handle, sl, ns, _stream(stream)))


def dot_product_matrix(field, rows, row_len: int, nrows: int, terms: Sequence, stream=None) -> None:
    """Overwrite form of mul_add_matrix (src/ops.rs:773-810)."""
    if _wide(field) and terms and all(len(c) == nrows for c, _ in terms):
        plan = Plan.matrix(field, len(terms), nrows, [int(v) for c, _ in terms for v in c])
        return dot_product_matrix_with(rows, row_len, nrows, plan, [src for _, src in terms], stream)
    r, rn = _buf(rows)
    arr, n, _keep = _terms(terms)
    check(lib().fgfc_dot_product_matrix(_fid(field), r, rn, row_len, nrows, arr, n, _stream(stream)))


def dot_product_matrix_with(rows, row_len: int, nrows: int, plan: Plan, srcs: Sequence,
                            stream=None) -> None:
    """The RS encode shape (src/ops.rs:823-867)."""
    r, rn = _buf(rows)
    sl, ns = _slices(srcs)
    check(lib().fgfc_dot_product_matrix_with(r, rn, row_len, nrows, plan.handle, sl, ns, _stream(stream)))


def mul_add_matrix_scattered(field, dst, row_len: int, row_starts: Sequence[int], terms: Sequence,
                             stream=None) -> None:
    """Rows at dst[row_starts[j]..] (src/ops.rs:887-941)."""
    if _wide(field) and terms and all(len(c) == len(row_starts) for c, _ in terms):
        plan = Plan.matrix(field, len(terms), len(row_starts), [int(v) for c, _ in terms for v in c])
        return mul_add_matrix_scattered_with(dst, row_len, row_starts, plan, [src for _, src in terms], stream)
    d, dn = _buf(dst)
    starts = (C.c_size_t * max(1, len(row_starts)))(*[int(s) for s in row_starts])
    arr, n, _keep = _terms(terms)
    check(lib().fgfc_mul_add_matrix_scattered(_fid(field), d, dn, row_len, starts, len(row_starts), arr, n,
                                              _stream(stream)))


def mul_add_matrix_scattered_with(dst, row_len: int, row_starts: Sequence[int], plan: Plan,
                                  srcs: Sequence, stream=None) -> None:
    """Extension (no reference counterpart): the scattered op driven by a
    prepared plan of dimensions (len(srcs), len(row_starts))."""
    d, dn = _buf(dst)
    starts = (C.c_size_t * max(1, len(row_starts)))(*[int(s) for s in row_starts])
    sl, ns = _slices(srcs)
    check(lib().fgfc_mul_add_matrix_scattered_with(d, dn, row_len, starts, len(row_starts), plan.handle, sl,
                                                   ns, _stream(stream)))


def dot_product_matrix_scattered_with(dst, row_len: int, row_starts: Sequence[int], plan: Plan,
                                      srcs: Sequence, stream=None) -> None:
    """Extension (no reference counterpart): the overwrite form of the
    scattered op. Equal to zeroing the rows, then mul_add_matrix_scattered."""
    d, dn = _buf(dst)
    starts = (C.c_size_t * max(1, len(row_starts)))(*[int(s) for s in row_starts])
    sl, ns = _slices(srcs)
    check(lib().fgfc_dot_product_matrix_scattered_with(d, dn, row_len, starts, len(row_starts), plan.handle,
                                                       sl, ns, _stream(stream)))


# ---------------------------------------------------------------- pack / unpack (host)

def pack(field, elems: Sequence[int]) -> bytes:
    """Stable little-endian encoding (src/ops.rs:963-979)."""
    b = field.BYTES
    return b"".join(int(e).to_bytes(b, "little") for e in elems)


def pack_to_vec(field, elems: Sequence[int]) -> bytes:
    return pack(field, elems)


def unpack(field, data: bytes) -> list[int]:
    """src/ops.rs:985-1001."""
    b = field.BYTES
    if len(data) % b:
        raise FgfError(1, f"unpack: src is {len(data)} bytes, not a whole number of {field.NAME} elements")
    return [int.from_bytes(data[i:i + b], "little") for i in range(0, len(data), b)]
