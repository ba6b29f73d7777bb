"""fgfc_batch_run_noalloc: the work-list kernels on a fixed device scratch
array, for callers that may not allocate device memory while they run.
Each call must give, byte for byte, what the allocating raw entry points
(fgfc_dot_product_matrix, fgfc_mul_add_matrix,
fgfc_mul_add_matrix_scattered) give on the same inputs and what the CPU
oracle gives, two calls in a row must not see each other's scratch, and the
calls must leave the device's free memory unchanged. Collected last on
purpose: it also has to pass after everything else has run in the same
process."""
import ctypes as C

import numpy as np
import pytest
import torch

from fgf_b200 import _lib, ops
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32
from oracle import orc

pytestmark = pytest.mark.gpu

SCRATCH = 8 << 20
ERR_LIMIT = 12
ERR_ARG = 11
MAX_ROWS = {Gf8D: 16, Gf16: 8, Gf32: 4}


def _job(field, coeffs, srcs, dst, row_len, nrows, overwrite, starts=None, keep=None):
    """An fgfc_noalloc_job over device tensors; `keep` holds the ctypes arrays alive."""
    carr = (C.c_uint32 * max(1, len(coeffs)))(*[int(c) for c in coeffs])
    sarr = (_lib.Slice * max(1, len(srcs)))(*[_lib.Slice(s.data_ptr(), s.numel()) for s in srcs])
    rarr = None
    if starts is not None:
        rarr = (C.c_size_t * max(1, len(starts)))(*starts)
    keep.extend([carr, sarr, rarr])
    return _lib.NoAllocJob(
        C.cast(carr, C.POINTER(C.c_uint32)), C.cast(sarr, C.POINTER(_lib.Slice)), len(srcs),
        dst.data_ptr(), dst.numel(), C.cast(rarr, C.POINTER(C.c_size_t)) if rarr is not None else None,
        nrows, row_len, 1 if overwrite else 0)


def _run(field, jobs, stream=0):
    arr = (_lib.NoAllocJob * max(1, len(jobs)))(*jobs)
    return _lib.lib().fgfc_batch_run_noalloc(field.ID, arr, len(jobs), stream)


def _stripes(field, specs, seed):
    """Device sources/destinations for (k, m, row_len, kind, skew) specs, plus
    the coefficient matrix of each (term-major: coeffs[t * m + j])."""
    rng = np.random.default_rng(seed)
    out = []
    for k, m, rl, kind, skew in specs:
        coeffs = [int(x) for x in rng.integers(0, 1 << (8 * field.BYTES), size=k * m, dtype=np.uint64)]
        stride = (rl + 64 + 15) // 16 * 16
        pool = torch.from_numpy(rng.integers(0, 256, size=k * stride + 64, dtype=np.uint8)).cuda()
        # skew 0: every row 16-byte aligned (vector path); otherwise mixed offsets
        offs = [t * stride + (skew + t % 3 if skew else 0) for t in range(k)]
        srcs = [pool[o:o + rl] for o in offs]
        if kind == "scatter":
            stride = rl + 3 * field.BYTES
            starts = [j * stride for j in range(m)][::-1]
            dst_n = stride * m
        else:
            starts = None
            dst_n = rl * m
        base = torch.from_numpy(rng.integers(0, 256, size=dst_n + 64, dtype=np.uint8)).cuda()
        dst = base[skew: skew + dst_n]
        out.append((k, m, rl, kind, coeffs, srcs, dst, starts))
    return out


def _expected(field, stripe):
    """The allocating raw entry point's result for one stripe, on a copy."""
    k, m, rl, kind, coeffs, srcs, dst, starts = stripe
    want = dst.clone()
    terms = [(coeffs[t * m:(t + 1) * m], srcs[t]) for t in range(k)]
    if kind == "scatter":
        ops.mul_add_matrix_scattered(field, want, rl, starts, terms)
    elif kind == "dot":
        ops.dot_product_matrix(field, want, rl, m, terms)
    else:
        ops.mul_add_matrix(field, want, rl, m, terms)
    return want


def _oracle(field, stripe):
    """The CPU oracle's result for one stripe (host arrays)."""
    k, m, rl, kind, coeffs, srcs, dst, starts = stripe
    out = dst.cpu().numpy().copy()
    hs = [s.cpu().numpy().copy() for s in srcs]
    if kind == "scatter":
        orc.mul_add_matrix_scattered(field.ID, out, rl, starts, coeffs, hs)
    elif kind == "dot":
        orc.dot_product_matrix(field.ID, out, rl, m, coeffs, hs)
    else:
        orc.mul_add_matrix(field.ID, out, rl, m, coeffs, hs)
    return out


CASES = {
    Gf8B: [
        (10, 4, 32768 + 16, "dot", 0),      # byte-table class, K = 10
        (14, 2, 4096 + 3, "scatter", 0),    # byte-table class, K = 14
        (16, 9, 3000, "add", 0),            # nibble class, 3 groups
    ],
    Gf8D: [
        (10, 4, 65536 + 5, "dot", 0),      # RS(10,4) encode shape
        (20, 16, 4099, "add", 0),          # most rows, sources processed in chunks
        (10, 4, 8192, "scatter", 0),       # reconstruct-style scattered rows
        (7, 3, 5001, "dot", 3),            # mixed alignments: scalar path only
        (64, 1, 1000, "add", 0),           # most sources
    ],
    Gf16: [
        (6, 8, 2 * 3001, "dot", 0),
        (5, 3, 2 * 700, "scatter", 0),
        (12, 5, 2 * 4096 + 6, "add", 2),
    ],
    Gf32: [
        (4, 4, 4 * 2049, "dot", 0),
        (9, 2, 4 * 333, "add", 4),
    ],
}


@pytest.mark.parametrize("field", [Gf8B, Gf8D, Gf16, Gf32], ids=lambda f: f.__name__)
def test_two_calls_in_a_row_match_the_allocating_entry_points(cuda, field):
    for call, seed in enumerate((11, 12)):
        stripes = _stripes(field, CASES[field], seed + 100 * field.ID)
        want = [_expected(field, s) for s in stripes]
        truth = [_oracle(field, s) for s in stripes]
        keep = []
        jobs = [_job(field, s[4], s[5], s[6], s[2], s[1], s[3] == "dot", s[7], keep) for s in stripes]
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = _run(field, jobs, torch.cuda.current_stream().cuda_stream)
        assert st == 0, _lib.lib().fgfc_last_error().decode()
        torch.cuda.synchronize()
        if call:  # the first call may load its kernels' code onto the device
            assert torch.cuda.mem_get_info()[0] == free_before, "the call changed the device's free memory"
        for i, (s, w, o) in enumerate(zip(stripes, want, truth)):
            assert torch.equal(s[6], w), f"call {call}, stripe {i} ({s[3]}, k={s[0]}, m={s[1]}) differs"
            assert np.array_equal(s[6].cpu().numpy(), o), f"call {call}, stripe {i} differs from the oracle"


def test_free_memory_unchanged_over_repeated_calls(cuda):
    stripes = _stripes(Gf8D, CASES[Gf8D], 21)
    keep = []
    jobs = [_job(Gf8D, s[4], s[5], s[6], s[2], s[1], s[3] == "dot", s[7], keep) for s in stripes]
    stream = torch.cuda.current_stream().cuda_stream
    assert _run(Gf8D, jobs, stream) == 0  # first call on this device: address lookup
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        assert _run(Gf8D, jobs, stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_a_capturing_stream_is_refused(cuda):
    stripes = _stripes(Gf8D, [(4, 2, 4096, "dot", 0)], 22)
    keep = []
    s = stripes[0]
    job = _job(Gf8D, s[4], s[5], s[6], s[2], s[1], True, None, keep)
    before = s[6].clone()
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=side):
        st = _run(Gf8D, [job], side.cuda_stream)
    assert st == ERR_ARG
    assert "captured" in _lib.lib().fgfc_last_error().decode()
    torch.cuda.synchronize()
    assert torch.equal(s[6], before)


def test_empty_and_zero_source_jobs(cuda):
    keep = []
    assert _run(Gf8D, []) == 0
    dst = torch.full((3 * 100,), 0x5A, dtype=torch.uint8, device="cuda")
    jobs = [_job(Gf8D, [], [], dst, 100, 3, True, None, keep)]  # empty sum overwrites with zero
    assert _run(Gf8D, jobs, torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    assert int(dst.count_nonzero()) == 0


def test_limits_are_rejected_before_any_work(cuda):
    keep = []
    lib = _lib.lib()
    for field, rows in MAX_ROWS.items():
        st = _stripes(field, [(2, rows + 1, 64 * field.BYTES, "add", 0)], 5)[0]
        before = st[6].clone()
        job = _job(field, st[4], st[5], st[6], st[2], st[1], False, None, keep)
        assert _run(field, [job]) == ERR_LIMIT
        assert "at most" in lib.fgfc_last_error().decode()
        torch.cuda.synchronize()
        assert torch.equal(st[6], before)
    # 65 sources
    st = _stripes(Gf8D, [(65, 1, 64, "add", 0)], 6)[0]
    assert _run(Gf8D, [_job(Gf8D, st[4], st[5], st[6], 64, 1, False, None, keep)]) == ERR_LIMIT
    # more scratch than the array holds: 300 stripes of 64 sources x 16 rows of tables
    st = _stripes(Gf8D, [(64, 16, 64, "add", 0)], 7)[0]
    job = _job(Gf8D, st[4], st[5], st[6], 64, 16, False, None, keep)
    assert _run(Gf8D, [job] * 300) == ERR_LIMIT
    msg = lib.fgfc_last_error().decode()
    assert "scratch" in msg and str(SCRATCH) in msg


def test_validation_matches_the_raw_forms(cuda):
    keep = []
    st = _stripes(Gf16, [(2, 2, 7, "dot", 0)], 8)[0]  # odd row length for a 2-byte field
    assert _run(Gf16, [_job(Gf16, st[4], st[5], st[6], 7, 2, True, None, keep)]) != 0
    assert "dot_product_matrix" in _lib.lib().fgfc_last_error().decode()
