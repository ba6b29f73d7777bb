"""ctypes binding of libfgfcuda.so (include/fgf_cuda.h).

The product path always goes through this library: there is no CPU
fallback, and a missing or unloadable library raises at first use.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("FGF_CUDA_LIB", _PKG / "libfgfcuda.so"))

c_size = C.c_size_t
c_u32 = C.c_uint32
c_u8p = C.c_void_p  # device pointers travel as integers
c_stream = C.c_void_p
c_status = C.c_int


class Term(C.Structure):
    """`fgfc_term`: one `(coeffs, src)` term of the many-to-many ops."""

    _fields_ = [("coeffs", C.POINTER(c_u32)), ("ncoeffs", c_size), ("src", c_u8p), ("src_len", c_size)]


class Slice(C.Structure):
    """`fgfc_slice`: a device source slice."""

    _fields_ = [("ptr", c_u8p), ("len", c_size)]


class MatrixJob(C.Structure):
    """`fgfc_matrix_job`: one stripe of a batched submission."""

    _fields_ = [
        ("plan", C.c_void_p),
        ("srcs", C.POINTER(Slice)),
        ("nsrcs", c_size),
        ("dst", c_u8p),
        ("dst_len", c_size),
        ("row_starts", C.POINTER(c_size)),
        ("nrows", c_size),
        ("row_len", c_size),
        ("overwrite", C.c_int),
    ]


class NoAllocJob(C.Structure):
    """fgfc_noalloc_job: one stripe of fgfc_batch_run_noalloc (raw coefficients)."""

    _fields_ = [
        ("coeffs", C.POINTER(C.c_uint32)),
        ("srcs", C.POINTER(Slice)),
        ("nsrcs", C.c_size_t),
        ("dst", C.c_void_p),
        ("dst_len", C.c_size_t),
        ("row_starts", C.POINTER(C.c_size_t)),
        ("nrows", C.c_size_t),
        ("row_len", C.c_size_t),
        ("overwrite", C.c_int),
    ]


class ServerConfig(C.Structure):
    """`fgfc_server_config`."""

    _fields_ = [
        ("hbm_budget", c_size),
        ("staging_bytes", c_size),
        ("max_batch", c_size),
        ("max_inflight", c_size),
        ("plan_cache", c_size),
        ("max_launch_bytes", c_size),
        ("plain", C.c_int),
        ("device", C.c_int),
    ]


class Request(C.Structure):
    """`fgfc_request`: one matrix call over host buffers."""

    _fields_ = [
        ("field", C.c_int),
        ("coeffs", C.POINTER(c_u32)),
        ("srcs", C.POINTER(Slice)),
        ("nsrcs", c_size),
        ("dst", C.c_void_p),
        ("dst_len", c_size),
        ("row_starts", C.POINTER(c_size)),
        ("nrows", c_size),
        ("row_len", c_size),
        ("overwrite", C.c_int),
    ]


class RebuildRequest(C.Structure):
    """`fgfc_rebuild_request`: a reconstruct by erasure pattern."""

    _fields_ = [
        ("field", C.c_int),
        ("parity", C.POINTER(c_u32)),
        ("k", c_size),
        ("m", c_size),
        ("survivors", C.POINTER(c_size)),
        ("srcs", C.POINTER(Slice)),
        ("erased", C.POINTER(c_size)),
        ("nerased", c_size),
        ("dst", C.c_void_p),
        ("dst_len", c_size),
        ("row_starts", C.POINTER(c_size)),
        ("row_len", c_size),
    ]


class ServerStats(C.Structure):
    """`fgfc_server_stats`."""

    _fields_ = [
        ("completed", C.c_uint64),
        ("failed", C.c_uint64),
        ("launches", C.c_uint64),
        ("plan_hits", C.c_uint64),
        ("plan_misses", C.c_uint64),
        ("source_bytes", C.c_uint64),
        ("peak_device_bytes", C.c_uint64),
        ("max_batch_seen", C.c_uint64),
        ("p50_us", C.c_double),
        ("p99_us", C.c_double),
        ("mean_us", C.c_double),
        ("max_us", C.c_double),
        ("busy_s", C.c_double),
        ("queue_us", C.c_double),
        ("launch_us", C.c_double),
    ]


_SIGS = {
    "fgfc_last_error": (C.c_char_p, []),
    "fgfc_version": (C.c_char_p, []),
    "fgfc_limits": (None, [C.POINTER(c_size), C.POINTER(c_size)]),
    "fgfc_field_bytes": (c_size, [C.c_int]),
    "fgfc_plan_create": (c_status, [C.c_int, c_size, c_size, C.POINTER(c_u32), C.POINTER(C.c_void_p)]),
    "fgfc_coeff_create": (c_status, [C.c_int, c_u32, C.POINTER(C.c_void_p)]),
    "fgfc_plan_destroy": (None, [C.c_void_p]),
    "fgfc_plan_dimensions": (c_status, [C.c_void_p, C.POINTER(c_size), C.POINTER(c_size)]),
    "fgfc_plan_len": (c_size, [C.c_void_p]),
    "fgfc_plan_field": (C.c_int, [C.c_void_p]),
    "fgfc_plan_values": (c_status, [C.c_void_p, C.POINTER(c_u32)]),
    "fgfc_plan_create_u64": (c_status, [C.c_int, c_size, c_size, C.POINTER(C.c_uint64), C.POINTER(C.c_void_p)]),
    "fgfc_coeff_create_u64": (c_status, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "fgfc_plan_values_u64": (c_status, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "fgfc_plan_get_at_u64": (c_status, [C.c_void_p, c_size, c_size, C.POINTER(C.c_uint64)]),
    "fgfc_plan_get_at": (c_status, [C.c_void_p, c_size, c_size, C.POINTER(c_u32)]),
    "fgfc_add_assign": (c_status, [C.c_int, c_u8p, c_size, c_u8p, c_size, c_stream]),
    "fgfc_mul_add": (c_status, [C.c_int, c_u8p, c_size, c_u32, c_u8p, c_size, c_stream]),
    "fgfc_mul_add_with": (c_status, [c_u8p, c_size, C.c_void_p, c_u8p, c_size, c_stream]),
    "fgfc_mul_into": (c_status, [C.c_int, c_u8p, c_size, c_u32, c_u8p, c_size, c_stream]),
    "fgfc_mul_into_with": (c_status, [c_u8p, c_size, C.c_void_p, c_u8p, c_size, c_stream]),
    "fgfc_mul_assign": (c_status, [C.c_int, c_u8p, c_size, c_u32, c_stream]),
    "fgfc_mul_assign_with": (c_status, [c_u8p, c_size, C.c_void_p, c_stream]),
    "fgfc_mul_elementwise": (c_status, [C.c_int, c_u8p, c_size, c_u8p, c_size, c_u8p, c_size, c_stream]),
    "fgfc_mul_add_scatter": (c_status, [C.c_int, c_u8p, c_size, c_size, C.POINTER(c_u32), c_size, c_u8p,
                                        c_size, c_stream]),
    "fgfc_mul_add_scatter_with": (c_status, [c_u8p, c_size, c_size, C.c_void_p, c_u8p, c_size, c_stream]),
    "fgfc_mul_add_gather": (c_status, [C.c_int, c_u8p, c_size, C.POINTER(c_u32), c_size, C.POINTER(Slice),
                                       c_size, c_stream]),
    "fgfc_mul_add_gather_with": (c_status, [c_u8p, c_size, C.c_void_p, C.POINTER(Slice), c_size, c_stream]),
    "fgfc_dot_product": (c_status, [C.c_int, c_u8p, c_size, C.POINTER(c_u32), c_size, C.POINTER(Slice),
                                    c_size, c_stream]),
    "fgfc_dot_product_with": (c_status, [c_u8p, c_size, C.c_void_p, C.POINTER(Slice), c_size, c_stream]),
    "fgfc_mul_add_matrix": (c_status, [C.c_int, c_u8p, c_size, c_size, c_size, C.POINTER(Term), c_size,
                                       c_stream]),
    "fgfc_mul_add_matrix_with": (c_status, [c_u8p, c_size, c_size, c_size, C.c_void_p, C.POINTER(Slice),
                                            c_size, c_stream]),
    "fgfc_dot_product_matrix": (c_status, [C.c_int, c_u8p, c_size, c_size, c_size, C.POINTER(Term), c_size,
                                           c_stream]),
    "fgfc_dot_product_matrix_with": (c_status, [c_u8p, c_size, c_size, c_size, C.c_void_p, C.POINTER(Slice),
                                                c_size, c_stream]),
    "fgfc_mul_add_matrix_scattered": (c_status, [C.c_int, c_u8p, c_size, c_size, C.POINTER(c_size), c_size,
                                                 C.POINTER(Term), c_size, c_stream]),
    "fgfc_mul_add_matrix_scattered_with": (c_status, [c_u8p, c_size, c_size, C.POINTER(c_size), c_size,
                                                      C.c_void_p, C.POINTER(Slice), c_size, c_stream]),
    "fgfc_dot_product_matrix_scattered_with": (c_status, [c_u8p, c_size, c_size, C.POINTER(c_size), c_size,
                                                          C.c_void_p, C.POINTER(Slice), c_size, c_stream]),
    "fgfc_cauchy_matrix": (c_status, [C.c_int, c_size, c_size, c_u32, C.POINTER(c_u32)]),
    "fgfc_decode_matrix": (c_status, [C.c_int, C.POINTER(c_u32), c_size, c_size, C.POINTER(c_size),
                                      C.POINTER(c_size), c_size, C.POINTER(c_u32)]),
    "fgfc_decode_plan_create": (c_status, [C.c_int, C.POINTER(c_u32), c_size, c_size, C.POINTER(c_size),
                                           C.POINTER(c_size), c_size, C.POINTER(C.c_void_p)]),
    "fgfc_batch_create": (c_status, [C.POINTER(C.c_void_p)]),
    "fgfc_batch_destroy": (None, [C.c_void_p]),
    "fgfc_batch_set_graphs": (c_status, [C.c_void_p, C.c_int]),
    "fgfc_batch_run": (c_status, [C.c_void_p, C.POINTER(MatrixJob), c_size, c_stream]),
    "fgfc_batch_stats": (c_status, [C.c_void_p, C.POINTER(c_size), C.POINTER(c_size), C.POINTER(C.c_int)]),
    "fgfc_batch_run_noalloc": (c_status, [C.c_int, C.POINTER(NoAllocJob), c_size, c_stream]),
    "fgfc_run_jobs_serial": (c_status, [C.POINTER(MatrixJob), c_size, c_stream]),
    "fgfc_device_check": (c_status, [C.c_int]),
    "fgfc_tune_force": (c_status, [C.c_int]),
    "fgfc_tune_choice": (C.c_int, [C.c_int, c_size, c_size, c_size]),
    "fgfc_tune_usable": (C.c_int, [C.c_int, C.c_int, c_size, c_size]),
    "fgfc_tune_shape": (c_status, [C.c_int, c_size, c_size, c_size, C.POINTER(C.c_int)]),
    "fgfc_tune_set_tile": (c_status, [c_size, c_size, C.c_uint]),
    "fgfc_tune_tile": (C.c_uint, [c_size, c_size]),
    "fgfc_tune_batch_tiles": (c_status, [C.c_void_p, C.POINTER(MatrixJob), c_size, c_stream,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fgfc_tune_save": (c_status, [C.c_char_p]),
    "fgfc_tune_load": (c_status, [C.c_char_p]),
    "fgfc_tune_clear": (None, []),
    "fgfc_server_create": (c_status, [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "fgfc_server_submit": (c_status, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "fgfc_server_submit_rebuild": (c_status, [C.c_void_p, C.POINTER(RebuildRequest), C.POINTER(C.c_uint64)]),
    "fgfc_server_wait": (c_status, [C.c_void_p, C.c_uint64]),
    "fgfc_server_poll": (c_status, [C.c_void_p, C.c_uint64, C.POINTER(C.c_int)]),
    "fgfc_server_drain": (c_status, [C.c_void_p]),
    "fgfc_server_get_stats": (c_status, [C.c_void_p, C.POINTER(ServerStats), C.c_int]),
    "fgfc_server_destroy": (None, [C.c_void_p]),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libfgfcuda.so once; raise if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"fgf_b200: CUDA library {LIB_PATH} is missing; build it with `python -m fgf_b200.build`")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


class FgfError(Exception):
    """A call the reference would reject with a panic.

    `status` is the fgfc_status code and `args[0]` the reference-style message.
    """

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int) -> None:
    if status != 0:
        msg = lib().fgfc_last_error().decode(errors="replace")
        raise FgfError(status, msg)
