"""Serving loop (`fgfc_server_*`).

No reference counterpart: fgf's callers issue one `ops` call per stripe on
the CPU. Each request here is exactly one such call -- `dot_product_matrix`
(overwrite), `mul_add_matrix` (accumulate) or `mul_add_matrix_scattered`
(src/ops.rs:675-941) -- over host memory (staged through page-locked
buffers) or device memory (used in place), validated the same way and
leaving the same bytes in the destination. The native worker admits requests in
arrival order against the device budget, runs each admitted group as one
batch launch, and overlaps copies and kernels of successive launches.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from ._lib import RebuildRequest, Request, ServerConfig, ServerStats, Slice, check, lib
from .ops import _fid


def _host(x) -> tuple[int, int, object]:
    """(address, byte length, owner) of a request buffer: numpy array, torch
    tensor (page-locked CPU tensors are copied without staging; CUDA tensors
    on the server's device are used in place), bytearray or (address,
    length). A request's buffers are all host memory or all device memory."""
    if isinstance(x, tuple):
        return int(x[0]), int(x[1]), None
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise TypeError("fgf_b200.serve: buffers must be contiguous")
        return int(x.data_ptr()), int(x.numel() * x.element_size()), x
    if hasattr(x, "ctypes"):
        if not x.flags["C_CONTIGUOUS"]:
            raise TypeError("fgf_b200.serve: buffers must be contiguous")
        return int(x.ctypes.data), int(x.nbytes), x
    if isinstance(x, bytearray):
        a = (C.c_uint8 * len(x)).from_buffer(x)
        return C.addressof(a), len(x), (x, a)
    raise TypeError(f"fgf_b200.serve: unsupported buffer type {type(x).__name__}")


class PreparedRequest:
    """A marshalled request; it can be submitted more than once (one at a time)."""

    def __init__(self, field, coeffs: Sequence[int], srcs: Sequence, dst, row_len: int, nrows: int,
                 overwrite: bool = True, row_starts: Sequence[int] | None = None):
        self.keep = []
        carr = (C.c_uint32 * max(1, len(coeffs)))(*[int(c) & 0xFFFFFFFF for c in coeffs])
        bufs = [_host(s) for s in srcs]
        sl = (Slice * max(1, len(bufs)))(*[Slice(p, n) for p, n, _ in bufs])
        d, dn, downer = _host(dst)
        rs = None
        if row_starts is not None:
            rs = (C.c_size_t * max(1, len(row_starts)))(*[int(v) for v in row_starts])
        self.keep = [carr, sl, rs, downer] + [o for _, _, o in bufs]
        self.source_bytes = len(bufs) * int(row_len)
        self.struct = Request(_fid(field), C.cast(carr, C.POINTER(C.c_uint32)), C.cast(sl, C.POINTER(Slice)),
                              len(bufs), d, dn, C.cast(rs, C.POINTER(C.c_size_t)) if rs is not None else None,
                              int(nrows), int(row_len), 1 if overwrite else 0)


class Server:
    """`fgfc_server`: continuous batching of requests over host or device buffers.

    `plain=True` serves one request at a time through the per-call entry
    points (the one-call-per-stripe comparison)."""

    def __init__(self, hbm_budget: int = 0, staging_bytes: int = 0, max_batch: int = 0, max_inflight: int = 0,
                 plan_cache: int = 0, max_launch_bytes: int = 0, plain: bool = False, device: int = -1):
        cfg = ServerConfig(hbm_budget, staging_bytes, max_batch, max_inflight, plan_cache, max_launch_bytes,
                           1 if plain else 0, device)
        h = C.c_void_p()
        check(lib().fgfc_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._live: dict[int, PreparedRequest] = {}

    def submit(self, field, coeffs: Sequence[int], srcs: Sequence, dst, row_len: int, nrows: int,
               overwrite: bool = True, row_starts: Sequence[int] | None = None) -> int:
        """Enqueue one call; its buffers must stay untouched until it completes."""
        return self.submit_prepared(PreparedRequest(field, coeffs, srcs, dst, row_len, nrows, overwrite,
                                                    row_starts))

    def submit_rebuild(self, field, parity: Sequence[Sequence[int]], survivors: Sequence[int], srcs: Sequence,
                       erased: Sequence[int], dst, row_len: int, row_starts: Sequence[int] | None = None) -> int:
        """Rebuild shards `erased` of the code [I_k ; parity] from the survivor
        shards `srcs` (indices `survivors`), written over dst; the server
        derives and caches the decode rows."""
        m, k = len(parity), len(survivors)
        flat = (C.c_uint32 * max(1, m * k))(*[int(v) for row in parity for v in row])
        sv = (C.c_size_t * max(1, k))(*[int(x) for x in survivors])
        er = (C.c_size_t * max(1, len(erased)))(*[int(x) for x in erased])
        bufs = [_host(x) for x in srcs]
        sl = (Slice * max(1, len(bufs)))(*[Slice(p, n) for p, n, _ in bufs])
        d, dn, downer = _host(dst)
        rs = None
        if row_starts is not None:
            rs = (C.c_size_t * max(1, len(row_starts)))(*[int(v) for v in row_starts])
        q = RebuildRequest(_fid(field), C.cast(flat, C.POINTER(C.c_uint32)), k, m, C.cast(sv, C.POINTER(C.c_size_t)),
                           C.cast(sl, C.POINTER(Slice)), C.cast(er, C.POINTER(C.c_size_t)), len(erased), d, dn,
                           C.cast(rs, C.POINTER(C.c_size_t)) if rs is not None else None, int(row_len))
        t = C.c_uint64()
        check(lib().fgfc_server_submit_rebuild(self._h, C.byref(q), C.byref(t)))
        keep = PreparedRequest.__new__(PreparedRequest)
        keep.keep = [flat, sv, er, sl, rs, downer] + [o for _, _, o in bufs]
        self._live[t.value] = keep
        return t.value

    def submit_prepared(self, req: PreparedRequest) -> int:
        t = C.c_uint64()
        check(lib().fgfc_server_submit(self._h, C.byref(req.struct), C.byref(t)))
        self._live[t.value] = req
        return t.value

    def wait(self, ticket: int) -> None:
        try:
            check(lib().fgfc_server_wait(self._h, ticket))
        finally:
            self._live.pop(ticket, None)

    def poll(self, ticket: int) -> bool:
        done = C.c_int()
        try:
            check(lib().fgfc_server_poll(self._h, ticket, C.byref(done)))
        except Exception:
            self._live.pop(ticket, None)
            raise
        if done.value:
            self._live.pop(ticket, None)
        return bool(done.value)

    def drain(self) -> None:
        check(lib().fgfc_server_drain(self._h))

    def stats(self, reset: bool = False) -> dict:
        s = ServerStats()
        check(lib().fgfc_server_get_stats(self._h, C.byref(s), 1 if reset else 0))
        return {name: getattr(s, name) for name, _ in ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            lib().fgfc_server_destroy(self._h)
            self._h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
