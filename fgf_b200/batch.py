"""Batched submissions of many stripes in one persistent launch per class.

No reference counterpart: the reference is a single-threaded CPU library
that serves one `ops` call at a time. A batch groups the arguments of many
`dot_product_matrix_with` / `mul_add_matrix_with` /
`mul_add_matrix_scattered_with` calls (src/ops.rs:720-941); each job is
validated exactly as that call would be, and the results are bit-identical
to issuing the calls one by one.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

from ._lib import MatrixJob, Slice, check, lib
from .ops import Plan, _buf, _stream


@dataclass
class Job:
    """One stripe: `plan` has dimensions (len(srcs), nrows)."""

    plan: Plan
    srcs: Sequence
    dst: object
    row_len: int
    nrows: int
    overwrite: bool = True
    row_starts: Sequence[int] | None = None  # scattered rows (overwrite: zero-then-accumulate in one pass)


class Prepared:
    """Marshalled job array; submit it repeatedly with `Batch.run_prepared`."""

    def __init__(self, jobs: Sequence[Job]):
        self.jobs = list(jobs)
        self._keep = []
        arr = (MatrixJob * max(1, len(self.jobs)))()
        for i, j in enumerate(self.jobs):
            bufs = [_buf(s) for s in j.srcs]
            sl = (Slice * max(1, len(bufs)))(*[Slice(p, n) for p, n in bufs])
            d, dn = _buf(j.dst)
            rs = None
            if j.row_starts is not None:
                rs = (C.c_size_t * max(1, len(j.row_starts)))(*[int(x) for x in j.row_starts])
            self._keep.extend([sl, rs])
            arr[i] = MatrixJob(j.plan.handle, C.cast(sl, C.POINTER(Slice)), len(bufs), d, dn,
                               C.cast(rs, C.POINTER(C.c_size_t)) if rs is not None else None,
                               j.nrows, j.row_len, 1 if j.overwrite else 0)
        self.array = arr
        self.n = len(self.jobs)


class Batch:
    """`fgfc_batch`: owns the device work-list, pinned staging and graphs."""

    def __init__(self, graphs: bool = True):
        h = C.c_void_p()
        check(lib().fgfc_batch_create(C.byref(h)))
        self._h = h
        check(lib().fgfc_batch_set_graphs(h, 1 if graphs else 0))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value:
            try:
                lib().fgfc_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    def prepare(self, jobs: Sequence[Job]) -> Prepared:
        return Prepared(jobs)

    def run(self, jobs: Sequence[Job], stream=None) -> None:
        self.run_prepared(Prepared(jobs), stream)

    def run_prepared(self, prepared: Prepared, stream=None) -> None:
        check(lib().fgfc_batch_run(self._h, prepared.array, prepared.n, _stream(stream)))

    def stats(self) -> dict:
        launches, items, rep = C.c_size_t(), C.c_size_t(), C.c_int()
        check(lib().fgfc_batch_stats(self._h, C.byref(launches), C.byref(items), C.byref(rep)))
        return {"launches": launches.value, "items": items.value, "graph_replayed": bool(rep.value)}


def run_serial(prepared: Prepared, stream=None) -> None:
    """Issue each job as its own per-call entry point (dot_product_matrix_with,
    mul_add_matrix_with or mul_add_matrix_scattered_with) from a native loop:
    the one-call-per-stripe baseline a batched submission replaces."""
    check(lib().fgfc_run_jobs_serial(prepared.array, prepared.n, _stream(stream)))
