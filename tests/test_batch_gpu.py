"""Batched submissions are bit-identical to the per-stripe calls they group."""
import numpy as np
import pytest
import torch

from fgf_b200 import batch as fb
from fgf_b200 import ops
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32
from oracle import orc

pytestmark = pytest.mark.gpu
noise = orc.noise


def d(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint8)).cuda()


def h(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def read(field, b):
    return ops.unpack(field, b.tobytes())


def _mixed_jobs(seed, pool):
    """Stripes of mixed field, k, m, length, alignment and mode, carved out
    of one device pool; returns (jobs, expected host results per job)."""
    host = h(pool)
    cursor = [0]

    def take(n, align=16, skew=0):
        c = (cursor[0] + align - 1) // align * align + skew
        cursor[0] = c + n + 64
        return c

    specs = [
        (Gf8D, 10, 4, 65536 + 7, True, None, 0),
        (Gf8D, 10, 4, 300000, True, None, 0),
        (Gf8B, 6, 3, 4096, False, None, 0),
        (Gf16, 5, 3, 2 * 3001, True, None, 0),
        (Gf16, 32, 8, 2 * 4096, True, None, 0),       # sources in chunks, rows in two passes
        (Gf32, 3, 2, 4 * 999, False, None, 0),
        (Gf32, 16, 4, 4 * 4096, True, None, 0),
        (Gf8D, 10, 4, 8192, False, "scatter", 0),      # reconstruct-style scattered rows
        (Gf8D, 4, 20, 5000, True, None, 0),           # 5 row groups -> 2 sub-jobs
        (Gf8D, 7, 2, 9999, True, None, 3),            # misaligned: whole stripe on the scalar path
        (Gf8B, 12, 1, 1 << 16, True, None, 0),
        (Gf8D, 20, 3, 7000, True, None, 0),           # Gf8 beyond the byte-table source limit
    ]
    jobs, expect = [], []
    for i, (field, k, m, rl, ovr, kind, skew) in enumerate(specs):
        b = field.BYTES
        coeffs = read(field, noise(k * m * b, seed + 10 * i))
        plan = ops.Plan.matrix(field, k, m, coeffs)
        s_off = [take(rl, skew=skew if t == 0 else 0) for t in range(k)]
        if skew:
            s_off = [o + (t % 3) for t, o in enumerate(s_off)]  # mixed alignments
        srcs_h = [host[o:o + rl].copy() for o in s_off]
        if kind == "scatter":
            gap = 3 * b
            stride = rl + gap
            d_off = take(stride * m)
            starts = [j * stride for j in range(m)][::-1]
            dst = pool[d_off:d_off + stride * m]
            want = host[d_off:d_off + stride * m].copy()
            orc.mul_add_matrix_scattered(field.ID, want, rl, starts, coeffs, srcs_h)
            jobs.append(fb.Job(plan, [pool[o:o + rl] for o in s_off], dst, rl, m, False, starts))
        else:
            d_off = take(rl * m, skew=skew)
            dst = pool[d_off:d_off + rl * m]
            want = host[d_off:d_off + rl * m].copy()
            if ovr:
                orc.dot_product_matrix(field.ID, want, rl, m, coeffs, srcs_h)
            else:
                orc.mul_add_matrix(field.ID, want, rl, m, coeffs, srcs_h)
            jobs.append(fb.Job(plan, [pool[o:o + rl] for o in s_off], dst, rl, m, ovr))
        expect.append((dst, want))
        assert cursor[0] < pool.numel()
    return jobs, expect


def test_batch_matches_oracle_mixed_geometry(cuda):
    pool = d(noise(24 << 20, 0xBA7C))
    jobs, expect = _mixed_jobs(0x100, pool)
    b = fb.Batch()
    b.run(jobs)
    for i, (dst, want) in enumerate(expect):
        assert np.array_equal(h(dst), want), f"job {i}"
    st = b.stats()
    assert st["launches"] >= 1 and st["items"] >= len(jobs)


def test_batch_graph_replay_uses_fresh_descriptors(cuda):
    """A repeated submission replays the captured graph, and new source bytes
    behind the same pointers are computed correctly each time."""
    k, m, rl = 10, 4, 3 * 65536 + 16 * 5
    coeffs = [int(x) for x in orc.cauchy(orc.GF8D, m, k).T.reshape(-1)]
    plan = ops.Plan.matrix(Gf8D, k, m, coeffs)
    nst = 6
    srcs = d(noise(nst * k * rl, 0x51))
    outs = d(np.zeros(nst * m * rl, np.uint8))
    jobs = [fb.Job(plan, [srcs[(s * k + t) * rl:(s * k + t + 1) * rl] for t in range(k)],
                   outs[s * m * rl:(s + 1) * m * rl], rl, m, True) for s in range(nst)]
    b = fb.Batch(graphs=True)
    prep = b.prepare(jobs)
    for rnd in range(6):
        data = noise(nst * k * rl, 0x52 + rnd)
        srcs.copy_(torch.from_numpy(data).cuda())
        b.run_prepared(prep)
        if rnd >= 4:  # each of the 4 descriptor slots captures once, then replays
            assert b.stats()["graph_replayed"]
        got = h(outs)
        for s in range(nst):
            want = np.zeros(m * rl, np.uint8)
            orc.dot_product_matrix(orc.GF8D, want, rl, m, coeffs,
                                   [data[(s * k + t) * rl:(s * k + t + 1) * rl] for t in range(k)])
            assert np.array_equal(got[s * m * rl:(s + 1) * m * rl], want), (rnd, s)


def test_batch_validation_and_empty_cases(cuda):
    b = fb.Batch()
    b.run([])
    plan = ops.Plan.matrix(Gf8D, 2, 3, [1, 2, 3, 4, 5, 6])
    dst = d(noise(3 * 64, 7))
    with pytest.raises(ops.FgfError, match="plan dimensions do not match"):
        b.run([fb.Job(plan, [dst[:64]], dst, 64, 3)])
    with pytest.raises(ops.FgfError, match="overlap"):
        b.run([fb.Job(plan, [dst[:16], dst[16:32]], dst, 16, 3, False, [0, 8, 40])])
    empty = ops.Plan.matrix(Gf8D, 0, 3, [])
    b.run([fb.Job(empty, [], dst, 64, 3, True)])
    assert not h(dst).any()


def test_batch_uniform_plan_with_tails_and_misalignment(cuda):
    """All stripes share one plan (the flattened grid-stride path): odd
    lengths, shared and mixed misalignment, overwrite and accumulate."""
    for field, k, m in ((Gf8D, 10, 4), (Gf8B, 3, 2), (Gf8D, 14, 1)):
        coeffs = read(field, noise(k * m, 0x77 + k))
        plan = ops.Plan.matrix(field, k, m, coeffs)
        pool = d(noise(8 << 20, 0x99 + k))
        host = h(pool)
        jobs, expect = [], []
        cur = 0
        for rl, skew, mixed, ovr in [(70001, 0, False, True), (4096, 5, False, True), (1000, 3, True, False),
                                     (65536 * 2 + 1, 0, False, False), (17, 0, False, True)]:
            offs = []
            for t in range(k):
                cur = (cur + 15) // 16 * 16 + skew + ((t % 3) if mixed else 0)
                offs.append(cur)
                cur += rl + 32
            cur = (cur + 15) // 16 * 16 + skew
            doff = cur
            cur += m * rl + 32
            want = host[doff:doff + m * rl].copy()
            srcs_h = [host[o:o + rl].copy() for o in offs]
            if ovr:
                orc.dot_product_matrix(field.ID, want, rl, m, coeffs, srcs_h)
            else:
                orc.mul_add_matrix(field.ID, want, rl, m, coeffs, srcs_h)
            dst = pool[doff:doff + m * rl]
            jobs.append(fb.Job(plan, [pool[o:o + rl] for o in offs], dst, rl, m, ovr))
            expect.append((dst, want))
        assert cur < pool.numel()
        b = fb.Batch()
        b.run(jobs)
        for i, (dst, want) in enumerate(expect):
            assert np.array_equal(h(dst), want), (field.NAME, k, m, i)


def test_batch_uniform_class_over_one_parameter_block(cuda):
    """More stripes than one launch parameter block holds (160) split into
    several launches of the same plan."""
    k, m, rl = 4, 2, 4096 + 12
    coeffs = read(Gf8D, noise(k * m, 0x31))
    plan = ops.Plan.matrix(Gf8D, k, m, coeffs)
    nst = 333
    data = noise(nst * k * rl, 0x32)
    srcs = d(data)
    outs = d(np.zeros(nst * m * rl, np.uint8))
    jobs = [fb.Job(plan, [srcs[(s * k + t) * rl:(s * k + t + 1) * rl] for t in range(k)],
                   outs[s * m * rl:(s + 1) * m * rl], rl, m, True) for s in range(nst)]
    b = fb.Batch()
    b.run(jobs)
    assert b.stats()["launches"] == 3
    got = h(outs)
    for s in (0, 159, 160, 161, 332):
        want = np.zeros(m * rl, np.uint8)
        orc.dot_product_matrix(orc.GF8D, want, rl, m, coeffs,
                               [data[(s * k + t) * rl:(s * k + t + 1) * rl] for t in range(k)])
        assert np.array_equal(got[s * m * rl:(s + 1) * m * rl], want), s


def test_tensor_core_bodies_in_a_batch(cuda):
    """Stripes given the tensor-core contraction (forced here: the built-in
    rule keeps it for the largest shapes only) run their 16-byte-aligned
    bodies as one launch per plan (several stripes of one plan share it) and
    their heads and tails on the table kernels. Every byte against the
    oracle, in two submissions with fresh data."""
    from fgf_b200 import tune

    with tune.forced("gf2mma"):
        _tensor_core_bodies_in_a_batch(tune)


def _tensor_core_bodies_in_a_batch(tune):
    rng = np.random.default_rng(91)
    specs = [  # field, k, m, row bytes, head offset, overwrite, scattered, plan id
        (Gf16, 32, 8, 2 * 150000 + 6, 0, True, False, 0),
        (Gf16, 32, 8, 2 * 131072, 0, True, False, 0),      # same plan: shares the launch
        (Gf16, 5, 3, 2 * 140003, 4, False, False, 1),      # unaligned head, accumulate
        (Gf8D, 10, 8, 300000 + 48, 0, True, True, 2),      # overwrite into scattered rows
        (Gf8B, 64, 16, 262144 + 1000, 0, True, False, 3),
        (Gf32, 16, 4, 4 * 70000, 8, True, False, 4),
        (Gf32, 7, 3, 4 * 80000, 0, False, True, 5),        # accumulate into scattered rows
    ]
    plans = {}
    for field, k, m, rl, hoff, ovr, sc, pid in specs:
        assert tune.chosen(field, k, m, rl) == "gf2mma", (field.__name__, k, m, rl)
        if pid not in plans:
            coeffs = [int(x) for x in rng.integers(0, 1 << (8 * field.BYTES), size=k * m, dtype=np.uint64)]
            plans[pid] = (coeffs, ops.Plan.matrix(field, k, m, coeffs))
    b = fb.Batch(graphs=True)
    for round_ in range(2):
        jobs, checks = [], []
        for field, k, m, rl, hoff, ovr, sc, pid in specs:
            coeffs, plan = plans[pid]
            stride = (rl + hoff + 64 + 255) // 256 * 256
            src_pool = d(rng.integers(0, 256, size=k * stride, dtype=np.uint8))
            srcs = [src_pool[t * stride + hoff:t * stride + hoff + rl] for t in range(k)]
            if sc:
                gap = (rl + 16 + 15) // 16 * 16 + 32
                dst = d(rng.integers(0, 256, size=gap * m + hoff + 16, dtype=np.uint8))[hoff:hoff + gap * m]
                starts = [j * gap for j in range(m)][::-1]
            else:
                dst = d(rng.integers(0, 256, size=rl * m + hoff + 16, dtype=np.uint8))[hoff:hoff + rl * m]
                starts = None
            want = h(dst).copy()
            hs = [h(x).copy() for x in srcs]
            if sc:
                if ovr:
                    for st in starts:
                        want[st:st + rl] = 0
                orc.mul_add_matrix_scattered(field.ID, want, rl, starts, coeffs, hs)
            elif ovr:
                orc.dot_product_matrix(field.ID, want, rl, m, coeffs, hs)
            else:
                orc.mul_add_matrix(field.ID, want, rl, m, coeffs, hs)
            jobs.append(fb.Job(plan, srcs, dst, rl, m, ovr, starts))
            checks.append((dst, want, srcs, src_pool))
        b.run(jobs)
        torch.cuda.synchronize()
        assert _lib_device_ok()
        for i, (dst, want, _, _) in enumerate(checks):
            got = h(dst)
            assert np.array_equal(got, want), f"round {round_}, stripe {i}: {int(np.count_nonzero(got != want))} bytes"


def _lib_device_ok():
    from fgf_b200 import _lib

    return _lib.lib().fgfc_device_check(1) == 0


@pytest.mark.parametrize("cols", [1, 2, 4, 16])
def test_every_tile_shape_gives_the_same_bytes(cuda, cols):
    """Work-list tile shapes (columns per thread per item) only change how the
    work is split: the mixed submission matches the oracle under each."""
    from fgf_b200 import tune
    try:
        for E in (1, 2, 4):
            for G in (1, 2, 3, 4):
                tune.set_tile(E, G, cols)
        pool = d(noise(24 << 20, 0xBA7D))
        jobs, expect = _mixed_jobs(0x200 + cols, pool)
        fb.Batch().run(jobs)
        for i, (dst, want) in enumerate(expect):
            assert np.array_equal(h(dst), want), f"job {i}, {cols} columns per thread"
    finally:
        tune.clear()


def test_tile_tuner_keeps_results_exact(cuda):
    """fgfc_tune_batch_tiles reruns an overwrite-only submission under each
    tile shape and keeps the fastest; the results stay bit-exact."""
    from fgf_b200 import tune
    rng = np.random.default_rng(0x711E)
    jobs, checks = [], []
    try:
        for i, (field, k, m, rl) in enumerate([(Gf16, 12, 8, 2 * 40000), (Gf16, 9, 3, 2 * 70001), (Gf8D, 20, 6, 90000),
                                               (Gf32, 7, 4, 4 * 30000), (Gf8D, 30, 2, 123457)]):
            vals = [int(x) for x in rng.integers(1, 1 << (8 * field.BYTES), size=k * m, dtype=np.uint64)]
            srcs_h = [noise(rl, 700 + 10 * i + t) for t in range(k)]
            want = np.zeros(m * rl, np.uint8)
            orc.dot_product_matrix(field.ID, want, rl, m, vals, srcs_h)
            dst = d(noise(m * rl, 799 + i))
            jobs.append(fb.Job(ops.Plan.matrix(field, k, m, vals), [d(x) for x in srcs_h], dst, rl, m, True))
            checks.append((dst, want))
        b = fb.Batch()
        before, after = tune.tune_batch_tiles(b, b.prepare(jobs))
        assert before > 0 and after > 0
        b.run(jobs)
        for i, (dst, want) in enumerate(checks):
            assert np.array_equal(h(dst), want), i
    finally:
        tune.clear()


@pytest.mark.parametrize("m", [3, 4, 7, 8, 11, 16])
def test_gf16_half_product_classes(cuda, m):
    """Gf16 stripes with 3, 4, 7 or 8 rows per 8-row sub-job run on byte
    half-products (lo = A + 0x20 B, hi = A + C): unaligned heads and ragged
    tails (scalar items), rows off the sources' 16-byte offset (shifted
    stores), accumulate and overwrite, more sources than one table pass."""
    rng = np.random.default_rng(0x16A + m)
    pool = d(noise(16 << 20, 0x16B + m))
    host = h(pool)
    jobs, checks = [], []
    cur = 256
    for i, (k, rl, src_skew, dst_skew, ovr, scattered) in enumerate([
            (5, 2 * 20011, 0, 0, True, False), (23, 2 * 9000 + 6, 4, 4, True, False),
            (12, 2 * 7777, 2, 10, False, False), (30, 2 * 4099, 0, 6, True, True), (3, 2 * 33, 6, 0, False, False)]):
        vals = [int(x) for x in rng.integers(0, 1 << 16, size=k * m, dtype=np.uint64)]
        s_off = []
        for t in range(k):
            s_off.append(cur + src_skew)
            cur += (rl + 64 + 255) // 256 * 256
        srcs_h = [host[o:o + rl].copy() for o in s_off]
        plan = ops.Plan.matrix(Gf16, k, m, vals)
        if scattered:
            stride = rl + 2 * 7
            base = cur + dst_skew
            cur += (stride * m + 511) // 256 * 256
            starts = [j * stride for j in range(m)][::-1]
            dst = pool[base:base + stride * m]
            want = host[base:base + stride * m].copy()
            if ovr:
                for j, st in enumerate(starts):
                    want[st:st + rl] = 0
            orc.mul_add_matrix_scattered(Gf16.ID, want, rl, starts, vals, srcs_h)
            jobs.append(fb.Job(plan, [pool[o:o + rl] for o in s_off], dst, rl, m, ovr, starts))
        else:
            base = cur + dst_skew
            cur += (rl * m + 511) // 256 * 256
            dst = pool[base:base + rl * m]
            want = host[base:base + rl * m].copy()
            (orc.dot_product_matrix if ovr else orc.mul_add_matrix)(Gf16.ID, want, rl, m, vals, srcs_h)
            jobs.append(fb.Job(plan, [pool[o:o + rl] for o in s_off], dst, rl, m, ovr))
        checks.append((dst, want))
        assert cur < pool.numel()
    fb.Batch().run(jobs)
    for i, (dst, want) in enumerate(checks):
        assert np.array_equal(h(dst), want), f"job {i}, m = {m}"
