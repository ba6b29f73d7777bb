"""Every C(14,4) = 1001 erasure pattern of the RS(10,4) Gf8D Cauchy code,
rebuilt on the device from decode plans made through the C ABI
(fgfc_decode_plan_create), all 1001 in one batched submission, each rebuilt
shard bit-exact against the original it replaces."""
from itertools import combinations

import numpy as np
import pytest
import torch

from fgf_b200 import batch as fb
from fgf_b200 import codes, ops
from fgf_b200.fields import Gf8D
from oracle import orc

pytestmark = pytest.mark.gpu


def test_rebuild_every_rs10_4_erasure_pattern(cuda):
    k, m, L = 10, 4, 4096 + 48
    c = codes.cauchy_matrix(Gf8D, m, k)
    vals = [c[i][t] for t in range(k) for i in range(m)]
    data = [orc.noise(L, 0xD0 + t) for t in range(k)]
    code = torch.zeros((k + m) * L, dtype=torch.uint8, device="cuda")
    for t in range(k):
        code[t * L:(t + 1) * L] = torch.from_numpy(data[t]).cuda()
    shards = [code[i * L:(i + 1) * L] for i in range(k + m)]
    ops.dot_product_matrix_with(code[k * L:], L, m, ops.Plan.matrix(Gf8D, k, m, vals), shards[:k])
    torch.cuda.synchronize()
    want_par = np.zeros(m * L, np.uint8)
    orc.dot_product_matrix(Gf8D.ID, want_par, L, m, vals, data)
    assert np.array_equal(code[k * L:].cpu().numpy(), want_par)

    patterns = list(combinations(range(k + m), m))
    assert len(patterns) == 1001
    out = torch.full((len(patterns) * m * L,), 0xEE, dtype=torch.uint8, device="cuda")
    plans, jobs = [], []
    for p, erased in enumerate(patterns):
        survivors = [i for i in range(k + m) if i not in erased][:k]
        plan = codes.decode_plan(Gf8D, c, survivors, list(erased))
        plans.append(plan)
        jobs.append(fb.Job(plan, [shards[s] for s in survivors], out[p * m * L:(p + 1) * m * L], L, m, True))
    b = fb.Batch()
    b.run(jobs)
    torch.cuda.synchronize()
    got = out.view(len(patterns), m, L)
    full = code.view(k + m, L)
    for p, erased in enumerate(patterns):
        assert torch.equal(got[p], full[list(erased)]), f"pattern {erased} not rebuilt"
