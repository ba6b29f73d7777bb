"""The serving loop: every request's result equals the single ops call it
stands for (checked against the oracle), whether it runs alone, in a mix of
requests batched together, or through plain one-call-per-request mode."""
import numpy as np
import pytest
import torch

from fgf_b200 import serve
from fgf_b200._lib import FgfError
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32
from oracle import orc

pytestmark = pytest.mark.gpu


def _buf(n, rng, pinned):
    a = rng.integers(0, 256, size=n, dtype=np.uint8)
    if pinned:
        t = torch.from_numpy(a).pin_memory()
        return t, t.numpy()
    return a, a


class Case:
    """One request: host sources and an initial destination, plus the oracle's answer."""

    def __init__(self, field, k, m, rl, kind, rng, pinned=False):
        self.field, self.k, self.m, self.rl, self.kind, self.pinned = field, k, m, rl, kind, pinned
        b = field.BYTES
        self.coeffs = [int(x) for x in rng.integers(0, 1 << (8 * b), size=k * m, dtype=np.uint64)]
        self.srcs = [_buf(rl, rng, pinned) for _ in range(k)]
        if kind == "scatter":
            stride = rl + 5 * b
            self.starts = [j * stride for j in range(m)][::-1]
            n = stride * m + 3 * b
        else:
            self.starts = None
            n = rl * m + 7  # surplus bytes past the rows must stay untouched
        self.init = rng.integers(0, 256, size=n, dtype=np.uint8)
        want = self.init.copy()
        sv = [v for _, v in self.srcs]
        if kind == "scatter":
            orc.mul_add_matrix_scattered(field.ID, want, rl, self.starts, self.coeffs, sv)
        elif kind == "dot":
            orc.dot_product_matrix(field.ID, want, rl, m, self.coeffs, sv)
        else:
            orc.mul_add_matrix(field.ID, want, rl, m, self.coeffs, sv)
        self.want = want

    def fresh_dst(self):
        if self.pinned:
            t = torch.from_numpy(self.init.copy()).pin_memory()
            return t, t.numpy()
        a = self.init.copy()
        return a, a

    def submit(self, srv, dst):
        return srv.submit(self.field, self.coeffs, [s for s, _ in self.srcs], dst, self.rl, self.m,
                          overwrite=self.kind == "dot", row_starts=self.starts)


def _cases(seed):
    rng = np.random.default_rng(seed)
    specs = [
        (Gf8D, 10, 4, 4 << 20, "dot", True),         # long first request: the rest queue behind it
        (Gf8D, 10, 4, 65536, "dot", False),
        (Gf8D, 10, 4, 4099, "scatter", False),
        (Gf8D, 20, 3, 7001, "add", False),
        (Gf8B, 6, 2, 333, "dot", False),
        (Gf16, 5, 3, 2 * 3001, "dot", False),
        (Gf16, 12, 5, 2 * 1000, "scatter", False),
        (Gf32, 4, 4, 4 * 999, "add", False),
        (Gf32, 3, 2, 4 * 257, "dot", False),
        (Gf8D, 10, 4, 300 << 10, "dot", True),       # page-locked, long rows: copied without staging
        (Gf8D, 10, 4, (256 << 10) + 3, "scatter", True),
        (Gf16, 8, 2, 2 * (200 << 10), "add", True),
        (Gf8D, 1, 1, 17, "dot", False),
        (Gf8D, 64, 1, 1000, "add", False),
    ]
    return [Case(f, k, m, rl, kind, rng, pinned) for f, k, m, rl, kind, pinned in specs]


def _check(cases, outs, label):
    for i, (c, (_, view)) in enumerate(zip(cases, outs)):
        assert np.array_equal(view, c.want), f"{label}: request {i} ({c.field.__name__}, {c.kind}, k={c.k}, " \
                                             f"m={c.m}, L={c.rl}) differs from the oracle"


def test_alone_in_the_mix_and_plain_give_the_oracle_result(cuda):
    cases = _cases(1)
    with serve.Server(hbm_budget=1 << 30, staging_bytes=256 << 20, max_inflight=1) as srv:
        alone = []
        for c in cases:
            d = c.fresh_dst()
            srv.wait(c.submit(srv, d[0]))
            alone.append(d)
        _check(cases, alone, "alone")
        srv.stats(reset=True)
        mix = [c.fresh_dst() for c in cases]
        tickets = [c.submit(srv, d[0]) for c, d in zip(cases, mix)]
        for t in tickets:
            srv.wait(t)
        _check(cases, mix, "mix")
        st = srv.stats()
        assert st["completed"] == len(cases) and st["failed"] == 0
        assert st["max_batch_seen"] >= 2 and st["launches"] < len(cases), st  # requests shared launches
        assert st["p99_us"] >= st["p50_us"] > 0
    with serve.Server(hbm_budget=1 << 30, staging_bytes=256 << 20, plain=True) as srv:
        plain = [c.fresh_dst() for c in cases]
        tickets = [c.submit(srv, d[0]) for c, d in zip(cases, plain)]
        srv.drain()
        for t in tickets:
            srv.wait(t)
        _check(cases, plain, "plain")
        assert srv.stats()["launches"] == len(cases)


def test_admission_keeps_device_use_within_the_budget(cuda):
    rng = np.random.default_rng(2)
    cases = [Case(Gf8D, 6, 3, 200000 + 16 * i, "dot", rng) for i in range(12)]  # ~1.8 MB on the device each
    budget = 4 << 20
    with serve.Server(hbm_budget=budget, staging_bytes=64 << 20) as srv:
        outs = [c.fresh_dst() for c in cases]
        tickets = [c.submit(srv, d[0]) for c, d in zip(cases, outs)]
        for t in tickets:
            srv.wait(t)
        _check(cases, outs, "budget")
        st = srv.stats()
        assert 0 < st["peak_device_bytes"] <= budget
        assert st["launches"] >= 6


def test_plan_cache_reuses_device_plans(cuda):
    rng = np.random.default_rng(3)
    base = Case(Gf16, 7, 3, 2 * 500, "dot", rng)
    with serve.Server(hbm_budget=64 << 20, staging_bytes=16 << 20) as srv:
        for _ in range(10):
            d = base.fresh_dst()
            srv.wait(base.submit(srv, d[0]))
            assert np.array_equal(d[1], base.want)
        st = srv.stats()
        assert st["plan_misses"] == 1 and st["plan_hits"] == 9


def test_limits_validation_and_trivial_requests(cuda):
    rng = np.random.default_rng(4)
    with serve.Server(hbm_budget=1 << 20, staging_bytes=1 << 20) as srv:
        big = Case(Gf8D, 4, 1, 300000, "dot", rng)
        with pytest.raises(FgfError) as e:
            big.submit(srv, big.fresh_dst()[0])
        assert e.value.status == 12
        src = np.zeros(7, np.uint8)
        with pytest.raises(FgfError) as e:
            srv.submit(Gf16, [1, 2], [src], np.zeros(14, np.uint8), 7, 2)
        assert e.value.status == 1 and "dot_product_matrix" in str(e.value)
        with pytest.raises(FgfError) as e:
            srv.submit(Gf8D, [1, 2], [np.zeros(8, np.uint8)], np.zeros(32, np.uint8), 8, 2, overwrite=False,
                       row_starts=[0, 4])
        assert e.value.status == 7 and "mul_add_matrix_scattered" in str(e.value)
        dst = np.full(30, 0x5A, np.uint8)
        srv.wait(srv.submit(Gf8D, [], [], dst, 10, 3))  # no sources: overwrite clears the rows
        assert not dst.any()
        dst = np.full(30, 0x5A, np.uint8)
        srv.wait(srv.submit(Gf8D, [], [], dst, 10, 3, overwrite=False))  # accumulate of nothing
        assert (dst == 0x5A).all()


def test_device_resident_requests_run_in_place(cuda):
    """Requests whose shards are already in device memory: no copies, same
    bytes as the oracle, alone, in the mix and in plain mode."""
    cases = _cases(5)[1:]
    for plain in (False, True):
        with serve.Server(hbm_budget=64 << 20, staging_bytes=16 << 20, plain=plain) as srv:
            for mode in ("alone", "mix"):
                dsrcs = [[torch.from_numpy(v.copy()).cuda() for _, v in c.srcs] for c in cases]
                dsts = [torch.from_numpy(c.init.copy()).cuda() for c in cases]
                tickets = []
                for c, ss, dd in zip(cases, dsrcs, dsts):
                    t = srv.submit(c.field, c.coeffs, ss, dd, c.rl, c.m, overwrite=c.kind == "dot",
                                   row_starts=c.starts)
                    if mode == "alone":
                        srv.wait(t)
                    else:
                        tickets.append(t)
                for t in tickets:
                    srv.wait(t)
                for i, (c, dd) in enumerate(zip(cases, dsts)):
                    assert np.array_equal(dd.cpu().numpy(), c.want), (plain, mode, i)
            st = srv.stats()
            assert st["peak_device_bytes"] == 0  # nothing was staged on the server's arena
    with serve.Server(hbm_budget=64 << 20, staging_bytes=16 << 20) as srv:
        with pytest.raises(FgfError) as e:
            srv.submit(Gf8D, [1], [torch.zeros(64, dtype=torch.uint8, device="cuda")], np.zeros(64, np.uint8), 64, 1)
        assert e.value.status == 11


def test_rebuild_requests_by_erasure_pattern(cuda):
    """fgfc_server_submit_rebuild: the server derives the decode rows of each
    pattern; rebuilt shards (written over garbage) equal the originals, for
    host and device buffers, alone and batched together."""
    from fgf_b200 import codes

    k, m, L = 10, 4, 65536 + 32
    parity = codes.cauchy_matrix(Gf8D, m, k)
    vals = [parity[i][t] for t in range(k) for i in range(m)]
    data = [orc.noise(L, 0xBE + t) for t in range(k)]
    shards = data + [np.zeros(L, np.uint8) for _ in range(m)]
    want = np.zeros(m * L, np.uint8)
    orc.dot_product_matrix(Gf8D.ID, want, L, m, vals, data)
    for j in range(m):
        shards[k + j] = want[j * L:(j + 1) * L].copy()
    rng = np.random.default_rng(77)
    patterns = [sorted(int(x) for x in rng.choice(k + m, size=m, replace=False)) for _ in range(12)]
    for where in ("host", "device"):
        srv = serve.Server(hbm_budget=1 << 30, staging_bytes=256 << 20)
        try:
            jobs = []
            for er in patterns:
                sv = [i for i in range(k + m) if i not in er][:k]
                if where == "host":
                    srcs = [shards[i] for i in sv]
                    out = np.full(m * L, 0xEE, np.uint8)
                else:
                    srcs = [torch.from_numpy(shards[i]).cuda() for i in sv]
                    out = torch.full((m * L,), 0xEE, dtype=torch.uint8, device="cuda")
                t = srv.submit_rebuild(Gf8D, parity, sv, srcs, er, out, L)
                jobs.append((t, er, out, srcs))
            for t, er, out, _ in jobs:
                srv.wait(t)
                got = out if where == "host" else out.cpu().numpy()
                for j, e in enumerate(er):
                    assert np.array_equal(got[j * L:(j + 1) * L], shards[e]), f"{where}: pattern {er} shard {e}"
            st = srv.stats()
            assert st["completed"] == len(patterns)
        finally:
            srv.close()


def test_overwrite_scattered_through_batch_and_single_call(cuda):
    """dot_product_matrix_scattered_with (batch job with row_starts and
    overwrite): equals zeroing the rows, then mul_add_matrix_scattered."""
    from fgf_b200 import batch as fb
    from fgf_b200 import ops

    rng = np.random.default_rng(78)
    for field, k, m, L in ((Gf8D, 10, 4, 65536 + 5), (Gf16, 6, 3, 2 * 5001), (Gf32, 4, 2, 4 * 1003)):
        coeffs = [int(x) for x in rng.integers(0, 1 << (8 * field.BYTES), size=k * m, dtype=np.uint64)]
        srcs_h = [rng.integers(0, 256, size=L, dtype=np.uint8) for _ in range(k)]
        gap = L + 3 * field.BYTES
        starts = [j * gap for j in range(m)][::-1]
        init = rng.integers(0, 256, size=gap * m + 8, dtype=np.uint8)
        want = init.copy()
        for st in starts:
            want[st:st + L] = 0
        orc.mul_add_matrix_scattered(field.ID, want, L, starts, coeffs, srcs_h)
        plan = ops.Plan.matrix(field, k, m, coeffs)
        srcs = [torch.from_numpy(s).cuda() for s in srcs_h]
        d1 = torch.from_numpy(init.copy()).cuda()
        ops.dot_product_matrix_scattered_with(d1, L, starts, plan, srcs)
        d2 = torch.from_numpy(init.copy()).cuda()
        fb.Batch().run([fb.Job(plan, srcs, d2, L, m, True, starts)])
        torch.cuda.synchronize()
        assert np.array_equal(d1.cpu().numpy(), want), field.__name__
        assert np.array_equal(d2.cpu().numpy(), want), field.__name__
