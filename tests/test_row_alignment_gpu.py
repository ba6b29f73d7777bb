"""Destination rows at any offset within 16 bytes. Contiguous rows of a
length that is not a multiple of 16 (the layout the reference's
`dot_product_matrix(rows, row_len, ..)` implies) put each row at a different
offset; the vector kernels splice their 16-byte columns across lanes for
such rows. Every byte must match the oracle, in every kernel family: the
single-call nibble kernel, the batch work-list kernels (nibble and byte
table) and the uniform-plan batch kernel."""
import numpy as np
import pytest
import torch

from fgf_b200 import batch as fb
from fgf_b200 import ops
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32
from oracle import orc

pytestmark = pytest.mark.gpu


def d(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint8)).cuda()


def h(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _coeffs(field, k, m, rng):
    return [int(x) for x in rng.integers(0, 1 << (8 * field.BYTES), size=k * m, dtype=np.uint64)]


def _expect(field, init, rl, m, coeffs, srcs, ovr):
    want = init.copy()
    if ovr:
        orc.dot_product_matrix(field.ID, want, rl, m, coeffs, srcs)
    else:
        orc.mul_add_matrix(field.ID, want, rl, m, coeffs, srcs)
    return want


@pytest.mark.parametrize("field", [Gf8D, Gf8B, Gf16, Gf32], ids=lambda f: f.__name__)
@pytest.mark.parametrize("k,m", [(3, 1), (10, 4), (5, 7), (14, 3)])
def test_single_call_contiguous_rows_of_every_residue(cuda, field, k, m):
    rng = np.random.default_rng(k * 100 + m + field.ID)
    b = field.BYTES
    for r in range(1, 16 // b):
        rl = 16 * 300 + r * b
        srcs = [rng.integers(0, 256, size=rl, dtype=np.uint8) for _ in range(k)]
        coeffs = _coeffs(field, k, m, rng)
        plan = ops.Plan.matrix(field, k, m, coeffs)
        ds = [d(s) for s in srcs]
        for ovr in (True, False):
            init = rng.integers(0, 256, size=rl * m + 5, dtype=np.uint8)
            want = _expect(field, init, rl, m, coeffs, srcs, ovr)
            got = d(init)
            if ovr:
                ops.dot_product_matrix_with(got[:rl * m], rl, m, plan, ds)
            else:
                ops.mul_add_matrix_with(got[:rl * m], rl, m, plan, ds)
            assert np.array_equal(h(got), want), (r, ovr)


@pytest.mark.parametrize("field,k,m", [(Gf8D, 10, 4), (Gf8B, 4, 2), (Gf8D, 20, 3), (Gf16, 6, 5), (Gf32, 5, 4)],
                         ids=lambda x: getattr(x, "__name__", str(x)))
@pytest.mark.parametrize("shared_plan", [True, False])
def test_batch_contiguous_rows_of_every_residue(cuda, field, k, m, shared_plan):
    """Many stripes in one submission: one shared plan (Gf8 with at most 4
    rows and 14 sources runs the uniform kernel) or one plan per stripe
    (work-list kernels)."""
    rng = np.random.default_rng(7 + k + m + field.ID + shared_plan)
    b = field.BYTES
    base_coeffs = _coeffs(field, k, m, rng)
    base_plan = ops.Plan.matrix(field, k, m, base_coeffs)
    jobs, checks = [], []
    for i, r in enumerate(list(range(1, 16 // b)) * 2):
        rl = 16 * (200 + 37 * i) + r * b
        coeffs = base_coeffs if shared_plan else _coeffs(field, k, m, rng)
        plan = base_plan if shared_plan else ops.Plan.matrix(field, k, m, coeffs)
        srcs = [rng.integers(0, 256, size=rl, dtype=np.uint8) for _ in range(k)]
        ovr = bool(i % 3)
        init = rng.integers(0, 256, size=rl * m, dtype=np.uint8)
        want = _expect(field, init, rl, m, coeffs, srcs, ovr)
        ds = [d(s) for s in srcs]
        got = d(init)
        jobs.append(fb.Job(plan, ds, got, rl, m, ovr))
        checks.append((got, want, plan, ds))
    bt = fb.Batch(graphs=False)
    bt.run(jobs)
    for i, (got, want, _, _) in enumerate(checks):
        assert np.array_equal(h(got), want), i
