"""The canonical Fan-Paar towers (src/field/fan_paar.rs) on the device path:
every op family against the CPU oracle, bit for bit (tolerance 0: the
arithmetic is exact). The kernels are field-agnostic: their tables come from
the images c * (single input bit) computed with the field's own product, so
these tests check that derivation for the tower X^2 + alpha X + 1 as well as
the device product of two varying operands (mul_elementwise)."""
import numpy as np
import pytest
import torch

from fgf_b200 import batch as fb
from fgf_b200 import ops, tune
from fgf_b200.fields import FanPaar8, FanPaar16, FanPaar32, cauchy, decode_rows, encode_plan_coeffs
from oracle import orc

pytestmark = pytest.mark.gpu

FP = [FanPaar8, FanPaar16, FanPaar32]
ids = lambda f: f.__name__  # noqa: E731


def d(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint8)).cuda()


def h(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def coeffs(field, n, rng, nonzero=False):
    lo = 1 if nonzero else 0
    return [int(x) for x in rng.integers(lo, 1 << (8 * field.BYTES), size=n, dtype=np.uint64)]


@pytest.mark.parametrize("field", FP, ids=ids)
def test_single_row_ops(cuda, field):
    rng = np.random.default_rng(0xFA + field.ID)
    for ln in (field.BYTES, 96, 4096 + 3 * field.BYTES):
        src, dst0 = orc.noise(ln, 11 + ln), orc.noise(ln, 12 + ln)
        for c in [0, 1] + coeffs(field, 3, rng, nonzero=True):
            got = d(dst0)
            ops.mul_add(field, got, c, d(src))
            want = dst0.copy()
            orc.mul_add(field.ID, want, c, src)
            assert np.array_equal(h(got), want), ("mul_add", ln, c)
            got = d(dst0)
            ops.mul_into(field, got, c, d(src))
            want = dst0.copy()
            orc.mul_into(field.ID, want, c, src)
            assert np.array_equal(h(got), want), ("mul_into", ln, c)
            got = d(dst0)
            ops.mul_assign(field, got, c)
            want = dst0.copy()
            orc.mul_assign(field.ID, want, c)
            assert np.array_equal(h(got), want), ("mul_assign", ln, c)


@pytest.mark.parametrize("field", FP, ids=ids)
def test_scatter_gather_dot(cuda, field):
    rng = np.random.default_rng(0xFB + field.ID)
    ln, m = 8192 + 4 * field.BYTES, 5
    src = orc.noise(ln, 21)
    rows0 = orc.noise(m * ln, 22)
    c = coeffs(field, m, rng)
    got = d(rows0)
    ops.mul_add_scatter(field, got, ln, c, d(src))
    want = rows0.copy()
    orc.mul_add_scatter(field.ID, want, ln, c, src)
    assert np.array_equal(h(got), want)
    srcs = [orc.noise(ln, 30 + t) for t in range(m)]
    dst0 = orc.noise(ln, 40)
    got = d(dst0)
    ops.mul_add_gather(field, got, c, [d(x) for x in srcs])
    want = dst0.copy()
    orc.mul_add_gather(field.ID, want, c, srcs)
    assert np.array_equal(h(got), want)
    got = d(dst0)
    ops.dot_product(field, got, c, [d(x) for x in srcs])
    want = dst0.copy()
    orc.dot_product(field.ID, want, c, srcs)
    assert np.array_equal(h(got), want)


@pytest.mark.parametrize("field", FP, ids=ids)
@pytest.mark.parametrize("k,m", [(10, 4), (3, 7), (16, 2)])
def test_matrix_ops_plan_and_raw(cuda, field, k, m):
    rng = np.random.default_rng(0xFC + 7 * k + m + field.ID)
    ln = 3 * 4096 + 8 * field.BYTES
    vals = coeffs(field, k * m, rng)
    srcs = [orc.noise(ln, 50 + t) for t in range(k)]
    rows0 = orc.noise(m * ln, 60)
    plan = ops.Plan.matrix(field, k, m, vals)
    for overwrite in (True, False):
        want = rows0.copy()
        (orc.dot_product_matrix if overwrite else orc.mul_add_matrix)(field.ID, want, ln, m, vals, srcs)
        got = d(rows0)
        (ops.dot_product_matrix_with if overwrite else ops.mul_add_matrix_with)(got, ln, m, plan, [d(x) for x in srcs])
        assert np.array_equal(h(got), want), ("plan", overwrite)
        got = d(rows0)
        terms = [(vals[t * m:(t + 1) * m], d(srcs[t])) for t in range(k)]
        (ops.dot_product_matrix if overwrite else ops.mul_add_matrix)(field, got, ln, m, terms)
        assert np.array_equal(h(got), want), ("raw", overwrite)


@pytest.mark.parametrize("field", FP, ids=ids)
def test_scattered_rows_and_unaligned_head(cuda, field):
    rng = np.random.default_rng(0xFD + field.ID)
    k, m, ln = 6, 3, 5000 * field.BYTES
    vals = coeffs(field, k * m, rng)
    pool = orc.noise((k + 1) * (ln + 64) + 16, 70)
    off = 4  # every source 4 bytes past a 16-byte boundary
    srcs_h = [pool[t * (ln + 64) + off:t * (ln + 64) + off + ln].copy() for t in range(k)]
    gap = ln + 48
    dst0 = orc.noise(gap * m + 64, 71)
    starts = [j * gap + 8 for j in range(m)][::-1]
    want = dst0.copy()
    orc.mul_add_matrix_scattered(field.ID, want, ln, starts, vals, srcs_h)
    got = d(dst0)
    dpool = d(pool)
    srcs = [dpool[t * (ln + 64) + off:t * (ln + 64) + off + ln] for t in range(k)]
    ops.mul_add_matrix_scattered(field, got, ln, starts, [(vals[t * m:(t + 1) * m], srcs[t]) for t in range(k)])
    assert np.array_equal(h(got), want)


@pytest.mark.parametrize("field", FP, ids=ids)
def test_elementwise(cuda, field):
    for ln in (0, field.BYTES, 33 * field.BYTES, 1 << 16):
        a, b = orc.noise(ln, 0x354), orc.noise(ln, 0x355)
        got = d(np.zeros(ln, np.uint8))
        if ln:
            ops.mul_elementwise(field, got, d(a), d(b))
        want = np.zeros(ln, np.uint8)
        orc.mul_elementwise(field.ID, want, a, b)
        assert np.array_equal(h(got), want), ln


@pytest.mark.parametrize("field,k,m", [(FanPaar8, 64, 16), (FanPaar16, 32, 8), (FanPaar32, 16, 4), (FanPaar16, 5, 3)],
                         ids=lambda x: getattr(x, "__name__", str(x)))
def test_tensor_core_contraction(cuda, field, k, m):
    rng = np.random.default_rng(0xFE + k)
    ln = 6 * 512 * field.BYTES + 4 * field.BYTES  # six 512-column blocks and a table-kernel tail
    vals = coeffs(field, k * m, rng)
    srcs = [orc.noise(ln, 80 + t) for t in range(k)]
    rows0 = orc.noise(m * ln, 90)
    want = rows0.copy()
    orc.dot_product_matrix(field.ID, want, ln, m, vals, srcs)
    with tune.forced("gf2mma"):
        got = d(rows0)
        ops.dot_product_matrix_with(got, ln, m, ops.Plan.matrix(field, k, m, vals), [d(x) for x in srcs])
        assert np.array_equal(h(got), want)


def test_batch_of_mixed_fields(cuda):
    """Fan-Paar stripes beside polynomial-field stripes in one submission."""
    from fgf_b200.fields import Gf8D, Gf16
    rng = np.random.default_rng(0xFF)
    jobs, checks = [], []
    for i, (field, k, m, ln) in enumerate([(FanPaar8, 10, 4, 65536 + 16), (FanPaar16, 8, 2, 40000), (Gf8D, 10, 4, 65536),
                                            (FanPaar32, 6, 3, 4 * 9000), (Gf16, 4, 2, 20000), (FanPaar8, 12, 6, 30000)]):
        vals = coeffs(field, k * m, rng)
        srcs_h = [orc.noise(ln, 100 * i + t) for t in range(k)]
        dst0 = orc.noise(m * ln, 100 * i + 99)
        want = dst0.copy()
        orc.dot_product_matrix(field.ID, want, ln, m, vals, srcs_h)
        dst = d(dst0)
        jobs.append(fb.Job(ops.Plan.matrix(field, k, m, vals), [d(x) for x in srcs_h], dst, ln, m, True))
        checks.append((dst, want))
    fb.Batch().run(jobs)
    torch.cuda.synchronize()
    for i, (dst, want) in enumerate(checks):
        assert np.array_equal(h(dst), want), i


@pytest.mark.parametrize("field", FP, ids=ids)
def test_erasure_round_trip(cuda, field):
    """Encode with a systematic Cauchy code over the field, erase as many
    shards as there are parity rows, rebuild them from the survivors."""
    k, m, ln = 6, 3, 8192 * field.BYTES
    c = cauchy(field, m, k)
    _, _, vals = encode_plan_coeffs(c)
    code = torch.zeros((k + m) * ln, dtype=torch.uint8, device="cuda")
    for t in range(k):
        code[t * ln:(t + 1) * ln] = d(orc.noise(ln, 500 + t))
    shards = [code[i * ln:(i + 1) * ln] for i in range(k + m)]
    ops.dot_product_matrix_with(code[k * ln:], ln, m, ops.Plan.matrix(field, k, m, vals), shards[:k])
    torch.cuda.synchronize()
    erased = [1, 4, 7]
    survivors = [i for i in range(k + m) if i not in erased][:k]
    truth = torch.stack([shards[e].clone() for e in erased])
    dm = decode_rows(field, c, survivors, erased)
    out = torch.full((m * ln,), 0x5A, dtype=torch.uint8, device="cuda")
    ops.dot_product_matrix_with(out, ln, m, ops.Plan.matrix(field, k, m, [dm[j][t] for t in range(k) for j in range(m)]),
                                [shards[s] for s in survivors])
    torch.cuda.synchronize()
    assert torch.equal(out.view(m, ln), truth)
