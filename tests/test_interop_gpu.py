"""Wire-format check for Gf8D (0x11D), the field fgf keeps so codecs above it
produce shards byte-identical to Intel ISA-L, klauspost/reedsolomon and the
classical Reed-Solomon tables (src/field/gf8d.rs:9-16).

Byte-identical shards follow from the same field (pinned to the reference's
0x11D known answers in tests/golden) and the same coding matrix. The matrices
of those ecosystems are restated here from their published constructions:

* Cauchy, ISA-L style: parity row i (k <= i < n), column j: inv(i ^ j);
  the library's fgfc_cauchy_matrix with x0 = k is exactly this matrix;
* Vandermonde, ISA-L style: parity row r holds g_r^j with g_0 = 1 and
  g_{r+1} = 2 * g_r;
* systematic Vandermonde (the Backblaze / klauspost construction): V[r][c] =
  r^c over n rows, multiplied by the inverse of its top k x k block, so the
  top k rows become the identity.

Every matrix is used through the device path (dot_product_matrix_with) and
compared with the oracle, and shards are rebuilt from every way of losing
m of them for the small code (RS(6,3)) to show the codes are MDS as used.
"""
from itertools import combinations

import numpy as np
import pytest
import torch

from fgf_b200 import batch as fb
from fgf_b200 import codes, ops
from fgf_b200.fields import Gf8D, invert, pow_
from oracle import orc

pytestmark = pytest.mark.gpu


def _cauchy_isal(k: int, m: int) -> list[list[int]]:
    return [[Gf8D.inv(i ^ j) for j in range(k)] for i in range(k, k + m)]


def _vandermonde_isal(k: int, m: int) -> list[list[int]]:
    rows, g = [], 1
    for _ in range(m):
        rows.append([pow_(Gf8D, g, j) for j in range(k)])
        g = Gf8D.mul(g, 2)
    return rows


def _systematic_vandermonde(k: int, m: int) -> list[list[int]]:
    n = k + m
    v = [[pow_(Gf8D, r, c) if (r or c) else 1 for c in range(k)] for r in range(n)]
    top_inv = invert(Gf8D, v[:k])
    full = [[0] * k for _ in range(n)]
    for r in range(n):
        for c in range(k):
            acc = 0
            for q in range(k):
                acc ^= Gf8D.mul(v[r][q], top_inv[q][c])
            full[r][c] = acc
    assert all(full[r][c] == (1 if r == c else 0) for r in range(k) for c in range(k))
    return full[k:]


def test_library_cauchy_is_the_isal_cauchy(cuda):
    for k, m in ((10, 4), (6, 3), (17, 5)):
        assert codes.cauchy_matrix(Gf8D, m, k, k) == _cauchy_isal(k, m)


@pytest.mark.parametrize("make", [_cauchy_isal, _vandermonde_isal, _systematic_vandermonde],
                         ids=["cauchy", "vandermonde", "systematic_vandermonde"])
@pytest.mark.parametrize("k,m", [(10, 4), (6, 3)])
def test_encode_and_rebuild_with_ecosystem_matrices(cuda, make, k, m):
    L = 8192 + 16
    parity = make(k, m)
    vals = [parity[i][t] for t in range(k) for i in range(m)]
    data = [orc.noise(L, 0x1D0 + 7 * t + k) for t in range(k)]
    code = torch.zeros((k + m) * L, dtype=torch.uint8, device="cuda")
    for t in range(k):
        code[t * L:(t + 1) * L] = torch.from_numpy(data[t]).cuda()
    shards = [code[i * L:(i + 1) * L] for i in range(k + m)]
    ops.dot_product_matrix_with(code[k * L:], L, m, ops.Plan.matrix(Gf8D, k, m, vals), shards[:k])
    torch.cuda.synchronize()
    want = np.zeros(m * L, np.uint8)
    orc.dot_product_matrix(Gf8D.ID, want, L, m, vals, data)
    assert np.array_equal(code[k * L:].cpu().numpy(), want)

    patterns = list(combinations(range(k + m), m))
    if len(patterns) > 120:
        rng = np.random.default_rng(k * 100 + m)
        patterns = [patterns[i] for i in rng.choice(len(patterns), size=120, replace=False)]
    jobs, plans, outs = [], [], []
    for er in patterns:
        sv = [i for i in range(k + m) if i not in er][:k]
        try:
            plan = codes.decode_plan(Gf8D, parity, sv, list(er))
        except Exception:
            pytest.fail(f"{make.__name__}: survivors {sv} do not determine the data (not MDS)")
        out = torch.full((m * L,), 0xEE, dtype=torch.uint8, device="cuda")
        plans.append(plan)
        outs.append(out)
        jobs.append(fb.Job(plan, [shards[s] for s in sv], out, L, m, True))
    fb.Batch().run(jobs)
    torch.cuda.synchronize()
    full = code.view(k + m, L)
    for er, out in zip(patterns, outs):
        assert torch.equal(out.view(m, L), full[list(er)]), f"{make.__name__}: pattern {er}"
