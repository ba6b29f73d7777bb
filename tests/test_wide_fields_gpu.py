"""The 8-byte fields, GF(2^64) (src/field/gf64.rs) and Fan-Paar GF(2^64)
(src/field/fan_paar.rs, fp64), on the device path: every op family against the
CPU oracle, bit for bit (tolerance 0: the arithmetic is exact), with 64-bit
coefficients that use the high word. The matrix ops run on the 8-byte table
kernel (wide.cu), whose tables come from the images c * (single input bit);
the raw forms prepare plans because the raw entry points take 32-bit values."""
import ctypes as C

import numpy as np
import pytest
import torch

from fgf_b200 import _lib
from fgf_b200 import batch as fb
from fgf_b200 import ops
from fgf_b200.fields import FanPaar64, Gf8D, Gf16, Gf64, cauchy, decode_rows, encode_plan_coeffs
from oracle import orc

pytestmark = pytest.mark.gpu

WIDE = [Gf64, FanPaar64]
ids = lambda f: f.__name__  # noqa: E731


def d(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint8)).cuda()


def h(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def coeffs(n, rng, nonzero=False):
    """Uniform 64-bit values; every one has a nonzero high word."""
    out = []
    for _ in range(n):
        v = int(rng.integers(1 << 32, 1 << 63, dtype=np.uint64)) | (int(rng.integers(0, 2)) << 63)
        out.append(v | (1 if nonzero else 0))
    return out


@pytest.mark.parametrize("field", WIDE, ids=ids)
def test_single_row_ops(cuda, field):
    rng = np.random.default_rng(0x640 + field.ID)
    for ln in (8, 96, 4096 + 24):
        src, dst0 = orc.noise(ln, 11 + ln), orc.noise(ln, 12 + ln)
        for c in [0, 1, 0xFFFFFFFF] + coeffs(3, rng, nonzero=True):
            for name in ("mul_add", "mul_into"):
                got = d(dst0)
                getattr(ops, name)(field, got, c, d(src))
                want = dst0.copy()
                getattr(orc, name)(field.ID, want, c, src)
                assert np.array_equal(h(got), want), (name, ln, hex(c))
                got = d(dst0)
                getattr(ops, name + "_with")(got, ops.Coeff(field, c), d(src))
                assert np.array_equal(h(got), want), (name + "_with", ln, hex(c))
            got = d(dst0)
            ops.mul_assign(field, got, c)
            want = dst0.copy()
            orc.mul_assign(field.ID, want, c)
            assert np.array_equal(h(got), want), ("mul_assign", ln, hex(c))


@pytest.mark.parametrize("field", WIDE, ids=ids)
def test_unaligned_sources_and_rows(cuda, field):
    """Sources and rows at offsets that are multiples of 8 bytes from nothing:
    the kernel's byte-wise load and store path."""
    rng = np.random.default_rng(0x641 + field.ID)
    ln = 8 * 3001
    pool = orc.noise(4 * ln + 64, 0x642)
    dpool = d(pool)
    for off in (1, 4, 12):
        c = coeffs(1, rng, nonzero=True)[0]
        src_h = pool[off:off + ln].copy()
        dst_h = pool[2 * ln + off + 8:3 * ln + off + 8].copy()
        want = dst_h.copy()
        orc.mul_add(field.ID, want, c, src_h)
        got_pool = dpool.clone()
        ops.mul_add(field, got_pool[2 * ln + off + 8:3 * ln + off + 8], c, got_pool[off:off + ln])
        assert np.array_equal(h(got_pool[2 * ln + off + 8:3 * ln + off + 8]), want), off


@pytest.mark.parametrize("field", WIDE, ids=ids)
def test_scatter_gather_dot(cuda, field):
    rng = np.random.default_rng(0x643 + field.ID)
    ln, m = 8192 + 8 * 3, 5
    src = orc.noise(ln, 21)
    rows0 = orc.noise(m * ln, 22)
    c = coeffs(m, rng)
    want = rows0.copy()
    orc.mul_add_scatter(field.ID, want, ln, c, src)
    got = d(rows0)
    ops.mul_add_scatter(field, got, ln, c, d(src))
    assert np.array_equal(h(got), want)
    got = d(rows0)
    ops.mul_add_scatter_with(got, ln, ops.Plan.new(field, c), d(src))
    assert np.array_equal(h(got), want)
    srcs = [orc.noise(ln, 30 + t) for t in range(m)]
    dst0 = orc.noise(ln, 40)
    for name in ("mul_add_gather", "dot_product"):
        want = dst0.copy()
        getattr(orc, name)(field.ID, want, c, srcs)
        got = d(dst0)
        getattr(ops, name)(field, got, c, [d(x) for x in srcs])
        assert np.array_equal(h(got), want), name
        got = d(dst0)
        getattr(ops, name + "_with")(got, ops.Plan.new(field, c), [d(x) for x in srcs])
        assert np.array_equal(h(got), want), name + "_with"


@pytest.mark.parametrize("field", WIDE, ids=ids)
@pytest.mark.parametrize("k,m", [(10, 4), (3, 7), (16, 2), (20, 12), (70, 1), (1, 9)])
def test_matrix_ops_plan_and_raw(cuda, field, k, m):
    """Shapes past the kernel's chunking: more than 8 rows (row chunks), more
    sources than one launch's shared-memory tables hold (later chunks
    accumulate), more than 64 sources."""
    rng = np.random.default_rng(0x644 + 7 * k + m + field.ID)
    ln = 2 * 4096 + 8 * 5
    vals = coeffs(k * m, rng)
    srcs = [orc.noise(ln, 50 + t) for t in range(k)]
    rows0 = orc.noise(m * ln, 60)
    plan = ops.Plan.matrix(field, k, m, vals)
    assert plan.values() == vals
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


@pytest.mark.parametrize("field", WIDE, ids=ids)
def test_scattered_rows(cuda, field):
    rng = np.random.default_rng(0x645 + field.ID)
    k, m, ln = 6, 3, 5000 * 8
    vals = coeffs(k * m, rng)
    pool = orc.noise((k + 1) * (ln + 64) + 16, 70)
    off = 4  # every source 4 bytes past a 16-byte boundary
    srcs_h = [pool[t * (ln + 64) + off:t * (ln + 64) + off + ln].copy() for t in range(k)]
    gap = ln + 48
    dst0 = orc.noise(gap * m + 64, 71)
    starts = [j * gap + 8 for j in range(m)][::-1]
    want = dst0.copy()
    orc.mul_add_matrix_scattered(field.ID, want, ln, starts, vals, srcs_h)
    dpool = d(pool)
    srcs = [dpool[t * (ln + 64) + off:t * (ln + 64) + off + ln] for t in range(k)]
    got = d(dst0)
    ops.mul_add_matrix_scattered(field, got, ln, starts, [(vals[t * m:(t + 1) * m], srcs[t]) for t in range(k)])
    assert np.array_equal(h(got), want)
    got = d(dst0)
    ops.mul_add_matrix_scattered_with(got, ln, starts, ops.Plan.matrix(field, k, m, vals), srcs)
    assert np.array_equal(h(got), want)


@pytest.mark.parametrize("field", WIDE, ids=ids)
def test_elementwise(cuda, field):
    for ln in (0, 8, 33 * 8, 1 << 16):
        a, b = orc.noise(ln, 0x646), orc.noise(ln, 0x647)
        got = d(np.zeros(ln, np.uint8))
        if ln:
            ops.mul_elementwise(field, got, d(a), d(b))
        want = np.zeros(ln, np.uint8)
        orc.mul_elementwise(field.ID, want, a, b)
        assert np.array_equal(h(got), want), ln


def test_elementwise_unaligned(cuda):
    ln = 8 * 777
    pool = orc.noise(3 * ln + 64, 0x648)
    dpool = d(pool)
    for field in WIDE:
        for off in (1, 8, 20):
            a, b = pool[off:off + ln], pool[ln + 32:2 * ln + 32]
            want = np.zeros(ln, np.uint8)
            orc.mul_elementwise(field.ID, want, a.copy(), b.copy())
            out = torch.zeros(ln + 16, dtype=torch.uint8, device="cuda")
            ops.mul_elementwise(field, out[off % 8:off % 8 + ln], dpool[off:off + ln], dpool[ln + 32:2 * ln + 32])
            assert np.array_equal(h(out[off % 8:off % 8 + ln]), want), (field.__name__, off)


def test_batch_with_wide_stripes(cuda):
    """8-byte stripes beside 1- and 2-byte stripes in one submission."""
    rng = np.random.default_rng(0x649)
    jobs, checks = [], []
    for i, (field, k, m, ln) in enumerate([(Gf64, 10, 4, 8 * 9000), (Gf8D, 10, 4, 65536), (FanPaar64, 6, 3, 8 * 5000),
                                            (Gf16, 4, 2, 20000), (Gf64, 3, 9, 8 * 700)]):
        if field.BYTES == 8:
            vals = coeffs(k * m, rng)
        else:
            vals = [int(x) for x in rng.integers(0, 1 << (8 * field.BYTES), size=k * m)]
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


@pytest.mark.parametrize("field", WIDE, ids=ids)
def test_erasure_round_trip(cuda, field):
    """Encode with a systematic Cauchy code over the field, erase as many
    shards as there are parity rows, rebuild them from the survivors."""
    k, m, ln = 6, 3, 8192 * 8
    c = cauchy(field, m, k)
    _, _, vals = encode_plan_coeffs(c)
    code = torch.zeros((k + m) * ln, dtype=torch.uint8, device="cuda")
    for t in range(k):
        code[t * ln:(t + 1) * ln] = d(orc.noise(ln, 500 + t))
    shards = [code[i * ln:(i + 1) * ln] for i in range(k + m)]
    ops.dot_product_matrix_with(code[k * ln:], ln, m, ops.Plan.matrix(field, k, m, vals), shards[:k])
    torch.cuda.synchronize()
    erased = [0, 4, 7]
    survivors = [i for i in range(k + m) if i not in erased][:k]
    truth = torch.stack([shards[e].clone() for e in erased])
    dm = decode_rows(field, c, survivors, erased)
    out = torch.full((m * ln,), 0x5A, dtype=torch.uint8, device="cuda")
    ops.dot_product_matrix_with(out, ln, m, ops.Plan.matrix(field, k, m, [dm[j][t] for t in range(k) for j in range(m)]),
                                [shards[s] for s in survivors])
    torch.cuda.synchronize()
    assert torch.equal(out.view(m, ln), truth)


def test_width_errors(cuda):
    """Lengths that are not whole 8-byte elements fail like the reference's
    width assertion; the 32-bit-coefficient entry points refuse the 8-byte
    fields with an error, never a wrong answer."""
    x = torch.zeros(12, dtype=torch.uint8, device="cuda")
    y = torch.zeros(12, dtype=torch.uint8, device="cuda")
    with pytest.raises(ops.FgfError):
        ops.mul_add(Gf64, x, 3 << 40, y)
    with pytest.raises(ops.FgfError):
        ops.mul_elementwise(FanPaar64, x, y, y)
    from fgf_b200 import codes
    with pytest.raises(ops.FgfError):
        codes.cauchy_matrix(Gf64, 2, 3)
    with pytest.raises(ops.FgfError):
        codes.decode_matrix(FanPaar64, [[1, 2, 3], [4, 5, 6]], [0, 1, 2], [3])
    st = _lib.lib().fgfc_batch_run_noalloc(Gf64.ID, C.cast(None, C.POINTER(_lib.NoAllocJob)), 0, None)
    assert st == 12  # FGFC_ERR_LIMIT
