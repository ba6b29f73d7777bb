"""Kernel-family choice (`fgfc_tune_*`): which kernel computes a matrix call.

A call runs the split-nibble table kernels, the byte-table kernels or the
bit-sliced tensor-core contraction; every family gives the same bytes. The
choice per (field, sources, rows, row-length bucket) is a process-wide
override, else a measured winner (`tune_shape`, persisted as JSON), else a
built-in rule.
"""
from __future__ import annotations

import contextlib
from typing import Iterator

from ._lib import check, lib
from .ops import _fid

AUTO, NIBBLE, BYTE, GF2MMA = 0, 1, 2, 3
NAMES = {AUTO: "auto", NIBBLE: "nibble", BYTE: "byte", GF2MMA: "gf2mma"}
IDS = {v: k for k, v in NAMES.items()}


def force(kernel: str | int) -> None:
    """Run every later call with this family where it can ("auto" restores the tuned choice)."""
    check(lib().fgfc_tune_force(IDS[kernel] if isinstance(kernel, str) else int(kernel)))


@contextlib.contextmanager
def forced(kernel: str | int) -> Iterator[None]:
    force(kernel)
    try:
        yield
    finally:
        force(AUTO)


def chosen(field, nsrcs: int, nrows: int, row_len: int) -> str:
    """The family a matrix call of this shape runs now."""
    return NAMES[lib().fgfc_tune_choice(_fid(field), nsrcs, nrows, row_len)]


def usable(kernel: str | int, field, nsrcs: int, nrows: int) -> bool:
    k = IDS[kernel] if isinstance(kernel, str) else int(kernel)
    return bool(lib().fgfc_tune_usable(k, _fid(field), nsrcs, nrows))


def variants_for(field, nsrcs: int, nrows: int, row_len: int) -> list[str]:
    """Every family that can run the shape, the current choice first."""
    first = chosen(field, nsrcs, nrows, row_len)
    rest = [n for k, n in NAMES.items() if k != AUTO and n != first and usable(k, field, nsrcs, nrows)]
    return [first] + rest


def tune_shape(field, nsrcs: int, nrows: int, row_len: int) -> str:
    """Measure the usable families on this shape and record the winner."""
    import ctypes as C

    out = C.c_int()
    check(lib().fgfc_tune_shape(_fid(field), nsrcs, nrows, row_len, C.byref(out)))
    return NAMES[out.value]


def set_tile(elem_bytes: int, groups: int, cols: int) -> None:
    """Element-vector columns per thread per work item of a batched
    split-nibble class (1, 2, 4, 8 or 16; 0 = built-in)."""
    check(lib().fgfc_tune_set_tile(elem_bytes, groups, cols))


def tile(elem_bytes: int, groups: int) -> int:
    return int(lib().fgfc_tune_tile(elem_bytes, groups))


def tune_batch_tiles(batch, prepared, stream=None) -> tuple[float, float]:
    """Measure tile shapes on one prepared submission (`batch.Batch`,
    `batch.Prepared`); returns its device time in microseconds with the
    starting and with the chosen tiles."""
    import ctypes as C

    from .ops import _stream

    before, after = C.c_double(), C.c_double()
    check(lib().fgfc_tune_batch_tiles(batch._h, prepared.array, prepared.n, _stream(stream), C.byref(before),
                                      C.byref(after)))
    return before.value, after.value


def save(path: str) -> None:
    check(lib().fgfc_tune_save(str(path).encode()))


def load(path: str) -> None:
    check(lib().fgfc_tune_load(str(path).encode()))


def clear() -> None:
    lib().fgfc_tune_clear()
