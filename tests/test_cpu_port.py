"""The CPU baseline (oracle/cpu_port.c, the restated AVX2+GFNI blocked
kernels) computes exactly what the scalar oracle computes, so the timed
baseline is doing the same work as the GPU path."""
import ctypes as C

import numpy as np
import pytest

from oracle import orc


class PortJob(C.Structure):
    _fields_ = [("field", C.c_int), ("k", C.c_size_t), ("m", C.c_size_t), ("row_len", C.c_size_t),
                ("coeffs", C.c_void_p), ("srcs", C.c_void_p), ("rows", C.c_void_p), ("overwrite", C.c_int)]


@pytest.fixture(scope="module")
def port():
    lib = orc.L()
    lib.orc_port_supported.restype = C.c_int
    lib.orc_port_job_size.restype = C.c_size_t
    if not lib.orc_port_supported():
        pytest.skip("host CPU lacks AVX2+GFNI")
    assert lib.orc_port_job_size() == C.sizeof(PortJob)
    return lib


MASK = [0xFF, 0xFF, 0xFFFF, 0xFFFFFFFF]


@pytest.mark.parametrize("field", [0, 1, 2, 3])
@pytest.mark.parametrize("k,m,rl,ovr", [(10, 4, 1000 * 4 + 36, 1), (3, 7, 256, 0), (1, 1, 100, 1),
                                        (5, 2, 4 * 33, 0), (16, 4, 4 * 512, 1)])
def test_port_matches_oracle(port, field, k, m, rl, ovr):
    srcs = [orc.noise(rl, 11 + t) for t in range(k)]
    co = (orc.noise(4 * k * m, 5 + field).view(np.uint32) & MASK[field]).astype(np.uint32)
    rows = [orc.noise(rl, 99 + j) for j in range(m)]
    want = np.concatenate(rows).copy()
    (orc.dot_product_matrix if ovr else orc.mul_add_matrix)(field, want, rl, m, co, srcs)
    sp = (C.c_void_p * k)(*[s.ctypes.data for s in srcs])
    rp = (C.c_void_p * m)(*[r.ctypes.data for r in rows])
    job = PortJob(field, k, m, rl, co.ctypes.data, C.cast(sp, C.c_void_p), C.cast(rp, C.c_void_p), ovr)
    port.orc_port_run_jobs(C.byref(job), C.c_size_t(1), 2)
    assert np.array_equal(np.concatenate(rows), want)
