"""Parity of the CUDA path with the oracle, mirroring the reference's
tests/ops.rs case by case (geometries, seeds, coefficient sweeps, the
surplus-row and gap checks). All results are bit-exact: the arithmetic is
GF(2^n), so the tolerance is zero."""
import numpy as np
import pytest
import torch

from fgf_b200 import ops
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32, FIELDS
from oracle import orc

pytestmark = pytest.mark.gpu

noise = orc.noise
LENGTHS = [0, 2, 8, 16, 18, 32, 34, 64, 66, 128, 254, 1024]  # tests/ops.rs:43


def d(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint8)).cuda()


def h(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def read(field, b: np.ndarray) -> list[int]:
    return ops.unpack(field, b.tobytes())


# ---------------------------------------------------------------- mul_add

@pytest.mark.parametrize("field", [Gf8B, Gf8D])
def test_gf8_mul_add_matches_oracle(cuda, field):
    # tests/ops.rs:48-61 and 1118-1130 (gf8d)
    for ln in LENGTHS:
        src = noise(ln, 0xA1)
        dsrc = d(src)
        base = noise(ln, 0xB2)
        got = d(np.tile(base, 256).reshape(256, ln)) if ln else None
        for c in range(256):
            if ln:
                ops.mul_add(field, got[c], c, dsrc)
        if ln:
            g = h(got)
            for c in range(256):
                want = base.copy()
                orc.mul_add(field.ID, want, c, src)
                assert np.array_equal(g[c], want), (ln, c)


def test_gf16_mul_add_matches_oracle(cuda):
    # tests/ops.rs:63-82
    coeffs = list(range(256)) + [i << 8 for i in range(256)] + [0x0108, 0x1234, 0xBEEF, 0xFFFF]
    for ln in LENGTHS:
        src = noise(ln, 0xC3)
        base = noise(ln, 0xD4)
        if not ln:
            continue
        dsrc = d(src)
        got = d(np.tile(base, len(coeffs)).reshape(len(coeffs), ln))
        for i, c in enumerate(coeffs):
            ops.mul_add(Gf16, got[i], c, dsrc)
        g = h(got)
        for i, c in enumerate(coeffs):
            want = base.copy()
            orc.mul_add(orc.GF16, want, c, src)
            assert np.array_equal(g[i], want), (ln, hex(c))


def test_mul_add_is_its_own_inverse(cuda):
    # tests/ops.rs:84-101
    src, original = noise(300, 0xE5), noise(300, 0xF6)
    for field, c in ((Gf8B, 0x8D), (Gf16, 0x9ACE)):
        b = d(original)
        ops.mul_add(field, b, c, d(src))
        assert not np.array_equal(h(b), original)
        ops.mul_add(field, b, c, d(src))
        assert np.array_equal(h(b), original)


# ---------------------------------------------------------------- mul_into / mul_assign

@pytest.mark.parametrize("field", [Gf8B, Gf8D])
def test_gf8_mul_into_and_mul_assign_agree(cuda, field):
    # tests/ops.rs:107-126, 1132-1146
    for ln in LENGTHS + [17]:
        if not ln:
            continue
        src = noise(ln, 0x11)
        into = d(np.full((256, ln), 0xAA, dtype=np.uint8))
        assign = d(np.tile(src, 256).reshape(256, ln))
        dsrc = d(src)
        for c in range(256):
            ops.mul_into(field, into[c], c, dsrc)
            ops.mul_assign(field, assign[c], c)
        gi, ga = h(into), h(assign)
        for c in range(256):
            want = np.zeros(ln, dtype=np.uint8)
            orc.mul_add(field.ID, want, c, src)
            assert np.array_equal(gi[c], want), ("into", ln, c)
            assert np.array_equal(ga[c], want), ("assign", ln, c)


def test_gf16_mul_into_and_mul_assign_agree(cuda):
    # tests/ops.rs:128-147
    for ln in LENGTHS:
        src = noise(ln, 0x22)
        for c in (0, 1, 0x0100, 0x0108, 0x00FF, 0xFF00, 0x1234, 0xFFFF):
            into = d(np.full(ln, 0xAA, dtype=np.uint8))
            assign = d(src)
            if ln:
                ops.mul_into(Gf16, into, c, d(src))
                ops.mul_assign(Gf16, assign, c)
            want = np.zeros(ln, dtype=np.uint8)
            orc.mul_add(orc.GF16, want, c, src)
            assert np.array_equal(h(into), want if ln else h(into))
            assert np.array_equal(h(assign), want)


def test_scaling_by_a_coefficient_then_its_inverse_is_identity(cuda):
    # tests/ops.rs:149-163
    original = noise(512, 0x33)
    for field, c in ((Gf8B, 0x57), (Gf16, 0x57A3), (Gf32, 0xDEADBEEF), (Gf8D, 0x57)):
        b = d(original)
        ops.mul_assign(field, b, c)
        ops.mul_assign(field, b, field.inv(c))
        assert np.array_equal(h(b), original)


def test_add_assign_is_xor_and_self_cancels(cuda):
    # tests/ops.rs:169-184
    for ln in LENGTHS:
        src, original = noise(ln, 0x44), noise(ln, 0x55)
        b = d(original)
        if ln:
            ops.add_assign(Gf8B, b, d(src))
            assert np.array_equal(h(b), original ^ src)
            ops.sub_assign(Gf8B, b, d(src))
        assert np.array_equal(h(b), original)


# ---------------------------------------------------------------- scatter / gather / matrix

def test_gf8_scatter_matches_repeated_mul_add(cuda):
    # tests/ops.rs:192-213
    for row_len in (1, 15, 16, 31, 32, 33, 64, 129, 512):
        for nrows in (1, 2, 3, 4, 5, 7, 8, 9):
            src = noise(row_len, 0x66)
            coeffs = [(j * 37) & 0xFF for j in range(nrows)]
            got0 = noise(row_len * nrows, 0x77)
            got = d(got0)
            ops.mul_add_scatter(Gf8B, got, row_len, coeffs, d(src))
            want = got0.copy()
            orc.mul_add_scatter(orc.GF8B, want, row_len, coeffs, src)
            assert np.array_equal(h(got), want), (row_len, nrows)


def test_gf16_scatter_matches_repeated_mul_add(cuda):
    # tests/ops.rs:215-236
    for row_len in (2, 16, 30, 32, 34, 64, 130, 512):
        for nrows in (1, 2, 3, 4, 5, 7, 8, 9):
            src = noise(row_len, 0x88)
            coeffs = [(j * 9871) & 0xFFFF for j in range(nrows)]
            got0 = noise(row_len * nrows, 0x99)
            got = d(got0)
            ops.mul_add_scatter(Gf16, got, row_len, coeffs, d(src))
            want = got0.copy()
            orc.mul_add_scatter(orc.GF16, want, row_len, coeffs, src)
            assert np.array_equal(h(got), want), (row_len, nrows)


@pytest.mark.parametrize("field,lens,cf", [
    (Gf8B, (1, 16, 33, 64, 100, 512), lambda t, j: ((t * 31 + j * 17) + 1) & 0xFF),
    (Gf16, (2, 16, 34, 64, 100, 512), lambda t, j: ((t * 7919 + j * 613) + 1) & 0xFFFF),
    (Gf8D, (1, 16, 33, 64, 100, 512), lambda t, j: ((t * 31 + j * 17) + 1) & 0xFF),
    (Gf32, (4, 16, 36, 64, 100, 512), lambda t, j: ((t * 0x9E3779B1 + j * 0x85EBCA77) + 1) & 0xFFFFFFFF),
])
def test_matrix_matches_repeated_scatter(cuda, field, lens, cf):
    # tests/ops.rs:238-300
    for row_len in lens:
        for nrows in (1, 2, 3, 4, 6, 8):
            for nterms in (1, 2, 5):
                sources = [noise(row_len, 0x100 + t) for t in range(nterms)]
                coeff_sets = [[cf(t, j) for j in range(nrows)] for t in range(nterms)]
                got0 = noise(row_len * nrows, 0xAA)
                got = d(got0)
                ops.mul_add_matrix(field, got, row_len, nrows,
                                   [(c, d(s)) for c, s in zip(coeff_sets, sources)])
                want = got0.copy()
                orc.mul_add_matrix(field.ID, want, row_len, nrows,
                                   [c for cs in coeff_sets for c in cs], sources)
                assert np.array_equal(h(got), want), (row_len, nrows, nterms)


def _check_dot_product_matrix(field, seed):
    # tests/ops.rs:314-385
    b = field.BYTES
    for rl_elems in (1, 16, 33, 64, 100, 512):
        row_len = rl_elems * b
        for nrows in (1, 2, 3, 4, 5, 6, 8):
            for nterms in (0, 1, 2, 5):
                sources = [noise(row_len, seed + 0x100 + t) for t in range(nterms)]
                coeff_sets = [read(field, noise(nrows * b, seed + 0x200 + t)) for t in range(nterms)]
                want = np.zeros(row_len * nrows, dtype=np.uint8)
                orc.dot_product_matrix(field.ID, want, row_len, nrows,
                                       [c for cs in coeff_sets for c in cs], sources)
                got0 = noise(row_len * (nrows + 1), seed + 0x300)
                got = d(got0)
                dsrc = [d(s) for s in sources]
                ops.dot_product_matrix(field, got, row_len, nrows, list(zip(coeff_sets, dsrc)))
                g = h(got)
                assert np.array_equal(g[:row_len * nrows], want), (row_len, nrows, nterms)
                assert np.array_equal(g[row_len * nrows:], got0[row_len * nrows:]), "surplus touched"
                if nterms:
                    flat = [c for cs in coeff_sets for c in cs]
                    plan = ops.Plan.matrix(field, nterms, nrows, flat)
                    prep = d(noise(row_len * nrows, seed + 0x500))
                    ops.dot_product_matrix_with(prep, row_len, nrows, plan, dsrc)
                    assert np.array_equal(h(prep), want), ("prepared", row_len, nrows, nterms)


@pytest.mark.parametrize("field,seed", [(Gf8B, 0x7A1), (Gf8D, 0x7A2), (Gf16, 0x7A3), (Gf32, 0x7A4)])
def test_dot_product_matrix_overwrites(cuda, field, seed):
    _check_dot_product_matrix(field, seed)


def _check_matrix_scattered(field, seed):
    # tests/ops.rs:410-469
    b = field.BYTES
    for rl_elems in (1, 16, 33, 64, 100, 512):
        row_len = rl_elems * b
        for nrows in (1, 2, 3, 4, 6, 8):
            for nterms in (1, 2, 5):
                sources = [noise(row_len, seed + 0x100 + t) for t in range(nterms)]
                coeff_sets = [read(field, noise(nrows * b, seed + 0x200 + t)) for t in range(nterms)]
                flat = [c for cs in coeff_sets for c in cs]
                init = noise(row_len * nrows, seed + 0x300)
                want = init.copy()
                orc.mul_add_matrix(field.ID, want, row_len, nrows, flat, sources)
                gap = b * 7
                stride = row_len + gap
                dst0 = noise(stride * nrows, seed + 0x400)
                starts = [j * stride for j in range(nrows)]
                for j in range(nrows):
                    dst0[starts[j]:starts[j] + row_len] = init[j * row_len:(j + 1) * row_len]
                dst = d(dst0)
                dsrc = [d(s) for s in sources]
                ops.mul_add_matrix_scattered(field, dst, row_len, starts, list(zip(coeff_sets, dsrc)))
                g = h(dst)
                for j in range(nrows):
                    assert np.array_equal(g[starts[j]:starts[j] + row_len],
                                          want[j * row_len:(j + 1) * row_len]), (row_len, nrows, nterms, j)
                    e = starts[j] + row_len
                    assert np.array_equal(g[e:e + gap], dst0[e:e + gap]), "gap modified"
                # the prepared extension agrees with the raw form
                plan = ops.Plan.matrix(field, nterms, nrows, flat)
                dst2 = d(dst0)
                ops.mul_add_matrix_scattered_with(dst2, row_len, starts, plan, dsrc)
                assert np.array_equal(h(dst2), g)


@pytest.mark.parametrize("field,seed", [(Gf8B, 0x5CA7), (Gf16, 0x5CA8), (Gf8D, 0x8D5C), (Gf32, 0x5CA9)])
def test_matrix_scattered_matches_contiguous(cuda, field, seed):
    _check_matrix_scattered(field, seed)


def test_matrix_scattered_pairs_coefficients_to_out_of_order_rows(cuda):
    # tests/ops.rs:481-499
    row_len = 64
    src = noise(row_len, 0x11)
    coeffs = [2, 9, 200]
    starts = [2 * row_len, row_len, 0]
    dst = d(np.zeros(3 * row_len, dtype=np.uint8))
    ops.mul_add_matrix_scattered(Gf8B, dst, row_len, starts, [(coeffs, d(src))])
    g = h(dst)
    for j, s in enumerate(starts):
        want = np.zeros(row_len, dtype=np.uint8)
        orc.mul_add(orc.GF8B, want, coeffs[j], src)
        assert np.array_equal(g[s:s + row_len], want)


def test_matrix_leaves_rows_beyond_nrows_untouched(cuda):
    # tests/ops.rs:526-537
    row_len = 64
    buf0 = noise(row_len * 8, 0xCC)
    b = d(buf0)
    ops.mul_add_matrix(Gf8B, b, row_len, 3, [([2, 3, 4], d(noise(row_len, 0xDD)))])
    assert np.array_equal(h(b)[row_len * 3:], buf0[row_len * 3:])


@pytest.mark.parametrize("field,n,coeffs,seed", [
    (Gf8B, 6, [0, 1, 0x53, 0xFF, 2, 0x1D], 0x300),
    (Gf16, 9, [0, 1, 0x0108, 0xFFFF, 2, 0x1D, 0x2000, 0xABCD, 0x0100], 0x340),
])
def test_gather_matches_summed_mul_add(cuda, field, n, coeffs, seed):
    # tests/ops.rs:539-570
    ln = 300
    sources = [noise(ln, seed + i) for i in range(n)]
    got0 = noise(ln, 0xEE if field is Gf8B else 0xEF)
    got = d(got0)
    ops.mul_add_gather(field, got, coeffs, [d(s) for s in sources])
    want = got0.copy()
    orc.mul_add_gather(field.ID, want, coeffs, sources)
    assert np.array_equal(h(got), want)


def test_dot_product_overwrites_and_matches_gather_from_zero(cuda):
    # tests/ops.rs:572-596
    ln = 96
    sources = [noise(ln, 0x348 + i) for i in range(6)]
    coeffs = [0, 1, 0x53, 0xFF, 2, 0x1D]
    want = np.zeros(ln, dtype=np.uint8)
    orc.mul_add_gather(orc.GF8B, want, coeffs, sources)
    initial = noise(ln, 0x34F)
    got = d(initial)
    ds = [d(s) for s in sources]
    ops.dot_product(Gf8B, got, coeffs, ds)
    assert np.array_equal(h(got), want)
    acc = d(initial)
    ops.mul_add_gather(Gf8B, acc, coeffs, ds)
    assert np.array_equal(h(acc) ^ initial, want)


def test_prepared_dot_product_matches_one_shot_over_gf16(cuda):
    # tests/ops.rs:598-619
    ln = 66
    sources = [noise(ln, 0x371), noise(ln, 0x372), noise(ln, 0x373)]
    ds = [d(s) for s in sources]
    coeffs = [0x0108, 0, 0xABCD]
    plan = ops.Plan(Gf16, coeffs)
    one = d(noise(ln, 0x374))
    prep = d(noise(ln, 0x375))
    ops.dot_product(Gf16, one, coeffs, ds)
    ops.dot_product_with(prep, plan, ds)
    assert np.array_equal(h(prep), h(one))
    single = d(noise(ln, 0x376))
    scaled = d(np.zeros(ln, dtype=np.uint8))
    ops.dot_product(Gf16, single, coeffs[:1], ds[:1])
    ops.mul_into(Gf16, scaled, coeffs[0], ds[0])
    assert np.array_equal(h(single), h(scaled))
    single_plan = ops.Plan(Gf16, coeffs[:1])
    sp = d(noise(ln, 0x377))
    ops.dot_product_with(sp, single_plan, ds[:1])
    assert np.array_equal(h(sp), h(scaled))


def test_empty_and_zero_dot_products_zero_the_destination(cuda):
    # tests/ops.rs:621-632
    e = d(noise(32, 0x377))
    ops.dot_product(Gf8B, e, [], [])
    assert not h(e).any()
    ds = [d(noise(32, 0x378)), d(noise(32, 0x379))]
    z = d(noise(32, 0x37A))
    ops.dot_product(Gf8B, z, [0, 0], ds)
    assert not h(z).any()


def test_prepared_coefficients_match_one_shot_operations(cuda):
    # tests/ops.rs:634-668
    src8 = noise(258, 0x350)
    for c in (0, 1, 2, 0x53, 0xFF):
        p = ops.Coeff(Gf8B, c)
        assert p.value() == c
        g0 = noise(258, 0x351)
        got, want = d(g0), d(g0)
        ops.mul_add_with(got, p, d(src8))
        ops.mul_add(Gf8B, want, c, d(src8))
        assert np.array_equal(h(got), h(want))
        got, want = d(np.zeros(258, np.uint8)), d(np.zeros(258, np.uint8))
        ops.mul_into_with(got, p, d(src8))
        ops.mul_into(Gf8B, want, c, d(src8))
        assert np.array_equal(h(got), h(want))
    src16 = noise(258, 0x352)
    for c in (0, 1, 2, 0x0108, 0xFFFF):
        p = ops.Coeff(Gf16, c)
        g0 = noise(258, 0x353)
        got, want = d(g0), d(g0)
        ops.mul_add_with(got, p, d(src16))
        ops.mul_add(Gf16, want, c, d(src16))
        assert np.array_equal(h(got), h(want))
        got, want = d(src16), d(src16)
        ops.mul_assign_with(got, p)
        ops.mul_assign(Gf16, want, c)
        assert np.array_equal(h(got), h(want))


def test_coefficient_plan_preserves_matrix_shape_and_reuses_entries(cuda):
    # tests/ops.rs:670-699
    values = [0, 1, 0x0108, 0xFFFF, 0x2000, 0xABCD]
    plan = ops.Plan.matrix(Gf16, 2, 3, values)
    assert plan.dimensions() == (2, 3)
    assert len(plan) == len(values) and not plan.is_empty()
    assert plan.values() == values
    assert plan.get(len(values)) is None
    coeff = plan.get(2)
    src = noise(258, 0x358)
    g0 = noise(258, 0x359)
    got, want = d(g0), d(g0)
    ops.mul_add_with(got, coeff, d(src))
    ops.mul_add(Gf16, want, values[2], d(src))
    assert np.array_equal(h(got), h(want))


def test_coefficient_plans_drive_all_multi_row_shapes(cuda):
    # tests/ops.rs:701-758
    row_len = 66
    coeffs = [0x0108, 0, 0xABCD]
    vp = ops.Plan(Gf16, coeffs)
    src = noise(row_len, 0x360)
    s0 = noise(row_len * 3, 0x361)
    a, b = d(s0), d(s0)
    ops.mul_add_scatter_with(a, row_len, vp, d(src))
    ops.mul_add_scatter(Gf16, b, row_len, coeffs, d(src))
    assert np.array_equal(h(a), h(b))
    sources = [noise(row_len, 0x362), noise(row_len, 0x363), noise(row_len, 0x364)]
    ds = [d(s) for s in sources]
    g0 = noise(row_len, 0x365)
    a, b = d(g0), d(g0)
    ops.mul_add_gather_with(a, vp, ds)
    ops.mul_add_gather(Gf16, b, coeffs, ds)
    assert np.array_equal(h(a), h(b))
    mv = [1, 0x0108, 2, 3, 0, 0xFFFF]
    mp = ops.Plan.matrix(Gf16, 2, 3, mv)
    m0 = noise(row_len * 3, 0x366)
    a, b = d(m0), d(m0)
    ops.mul_add_matrix_with(a, row_len, 3, mp, ds[:2])
    ops.mul_add_matrix(Gf16, b, row_len, 3, [(mv[:3], ds[0]), (mv[3:], ds[1])])
    assert np.array_equal(h(a), h(b))
    assert mp.get_at(1, 2).value() == mv[5]
    assert [c.value() for c in mp.row(1)] == mv[3:]


@pytest.mark.parametrize("field,row_len,seed", [(Gf8B, 79, 0x370), (Gf16, 78, 0x380), (Gf8D, 79, 0x390),
                                                (Gf32, 76, 0x3A0)])
def test_blocked_plans_match_raw_operations_across_group_boundaries(cuda, field, row_len, seed):
    # tests/ops.rs:760-820 (5 rows x 9 terms)
    NROWS, NTERMS = 5, 9
    values = read(field, noise(NROWS * NTERMS * field.BYTES, seed))
    values[0], values[1] = 0, 1
    vp = ops.Plan(field, values[:NROWS])
    src = noise(row_len, seed + 1)
    s0 = noise(row_len * NROWS, seed + 2)
    a, b = d(s0), d(s0)
    ops.mul_add_scatter_with(a, row_len, vp, d(src))
    ops.mul_add_scatter(field, b, row_len, values[:NROWS], d(src))
    want = s0.copy()
    orc.mul_add_scatter(field.ID, want, row_len, values[:NROWS], src)
    assert np.array_equal(h(a), want) and np.array_equal(h(b), want)
    gs = [noise(row_len, seed + 10 + i) for i in range(NROWS)]
    g0 = noise(row_len, seed + 20)
    a, b = d(g0), d(g0)
    ops.mul_add_gather_with(a, vp, [d(x) for x in gs])
    ops.mul_add_gather(field, b, values[:NROWS], [d(x) for x in gs])
    want = g0.copy()
    orc.mul_add_gather(field.ID, want, values[:NROWS], gs)
    assert np.array_equal(h(a), want) and np.array_equal(h(b), want)
    mp = ops.Plan.matrix(field, NTERMS, NROWS, values)
    ms = [noise(row_len, seed + 30 + i) for i in range(NTERMS)]
    m0 = noise(row_len * NROWS, seed + 40)
    a, b = d(m0), d(m0)
    ops.mul_add_matrix_with(a, row_len, NROWS, mp, [d(x) for x in ms])
    ops.mul_add_matrix(field, b, row_len, NROWS,
                       [(values[t * NROWS:(t + 1) * NROWS], d(ms[t])) for t in range(NTERMS)])
    want = m0.copy()
    orc.mul_add_matrix(field.ID, want, row_len, NROWS, values, ms)
    assert np.array_equal(h(a), want) and np.array_equal(h(b), want)


@pytest.mark.parametrize("field", [Gf8B, Gf8D, Gf16, Gf32])
def test_elementwise_products_match_field_arithmetic(cuda, field):
    # tests/ops.rs:840-879
    for ln in LENGTHS:
        if ln % field.BYTES:
            continue
        a, b = noise(ln, 0x354), noise(ln, 0x355)
        got = d(np.zeros(ln, np.uint8))
        if ln:
            ops.mul_elementwise(field, got, d(a), d(b))
        want = np.zeros(ln, np.uint8)
        orc.mul_elementwise(field.ID, want, a, b)
        assert np.array_equal(h(got), want), ln


@pytest.mark.parametrize("field", [Gf8B, Gf8D, Gf16, Gf32])
@pytest.mark.parametrize("offsets", [(0, 0, 0), (4, 4, 4), (1, 1, 1), (2, 2, 2), (0, 3, 8)],
                         ids=["aligned", "same4", "same1", "same2", "mixed"])
def test_elementwise_alignments_and_long_rows(cuda, field, offsets):
    """The kernel runs 16-byte vectors when dst, a and b share their offset
    within 16 bytes and the bytes before the first boundary are whole
    elements, and one element per step otherwise (and for heads and tails)."""
    rng = np.random.default_rng(0xE1 + field.ID)
    for ln in (field.BYTES, 7 * field.BYTES, 4096 + 3 * field.BYTES, (1 << 20) + 5 * field.BYTES):
        a_h = rng.integers(0, 256, size=ln, dtype=np.uint8)
        b_h = rng.integers(0, 256, size=ln, dtype=np.uint8)
        a_h[:min(ln, 8)] = 0  # zero operands
        pool = torch.zeros(3 * (ln + 64), dtype=torch.uint8, device="cuda")
        views = [pool[i * (ln + 64) + o:i * (ln + 64) + o + ln] for i, o in enumerate(offsets)]
        views[1].copy_(torch.from_numpy(a_h))
        views[2].copy_(torch.from_numpy(b_h))
        ops.mul_elementwise(field, views[0], views[1], views[2])
        want = np.zeros(ln, np.uint8)
        orc.mul_elementwise(field.ID, want, a_h, b_h)
        assert np.array_equal(h(views[0]), want), (ln, offsets)


def test_zero_and_one_coefficients_behave(cuda):
    # tests/ops.rs:881-895
    ln = 96
    src, original = noise(ln, 0xF0), noise(ln, 0x0F)
    b = d(original)
    ops.mul_add(Gf8B, b, 0, d(src))
    assert np.array_equal(h(b), original)
    ops.mul_add(Gf8B, b, 1, d(src))
    assert np.array_equal(h(b), original ^ src)
    b = d(original)
    ops.mul_assign(Gf16, b, 0)
    assert not h(b).any()


def test_erasure_round_trip_gf8(cuda):
    # tests/ops.rs:897-950: Vandermonde-style parity, 2 erasures, Cramer.
    k, m, row_len = 6, 3, 1024
    data = noise(k * row_len, 0x5150)
    g = Gf8B.GENERATOR

    def coeff(i, j):
        r = 1
        for _ in range((i + 1) * (j + 1)):
            r = Gf8B.mul(r, g)
        return r

    parity = d(np.zeros(m * row_len, np.uint8))
    dd = d(data)
    for i in range(k):
        ops.mul_add_scatter(Gf8B, parity, row_len, [coeff(i, j) for j in range(m)],
                            dd[i * row_len:(i + 1) * row_len])
    lost = [1, 4]
    residual = parity[:2 * row_len].clone()
    for i in (i for i in range(k) if i not in lost):
        ops.mul_add_matrix(Gf8B, residual, row_len, 2, [([coeff(i, 0), coeff(i, 1)],
                                                         dd[i * row_len:(i + 1) * row_len])])
    a0, b0 = coeff(lost[0], 0), coeff(lost[1], 0)
    a1, b1 = coeff(lost[0], 1), coeff(lost[1], 1)
    det = Gf8B.mul(a0, b1) ^ Gf8B.mul(a1, b0)
    assert det != 0
    di = Gf8B.inv(det)
    r0, r1 = residual[:row_len], residual[row_len:]
    x = d(np.zeros(row_len, np.uint8))
    y = d(np.zeros(row_len, np.uint8))
    ops.mul_add_gather(Gf8B, x, [Gf8B.mul(b1, di), Gf8B.mul(b0, di)], [r0, r1])
    ops.mul_add_gather(Gf8B, y, [Gf8B.mul(a1, di), Gf8B.mul(a0, di)], [r0, r1])
    assert np.array_equal(h(x), data[lost[0] * row_len:(lost[0] + 1) * row_len])
    assert np.array_equal(h(y), data[lost[1] * row_len:(lost[1] + 1) * row_len])


def test_empty_buffers_are_no_ops(cuda):
    # tests/ops.rs:1008-1017
    e = d(np.zeros(0, np.uint8))
    ops.mul_add(Gf8B, e, 7, e)
    ops.mul_assign(Gf16, e, 7)
    ops.mul_add_scatter(Gf8B, e, 0, [], e)
    ops.mul_add_matrix(Gf8B, e, 8, 0, [])
    ops.dot_product_matrix(Gf8B, e, 8, 0, [])
    ops.mul_add_gather(Gf8B, e, [], [])
    torch.cuda.synchronize()


@pytest.mark.parametrize("field,coeffs", [
    (Gf32, [0, 1, 0xDEADBEEF]),
    (Gf8D, [0, 1, 0x53, 0xFF, 0x02]),
])
def test_wide_field_ops(cuda, field, coeffs):
    # tests/ops.rs:1019-1108 check_wide_field_ops
    row_len = field.BYTES * 17
    s0, s1 = noise(row_len, 0x3200 + 8 * field.BYTES), noise(row_len, 0x6400 + 8 * field.BYTES)
    g0 = noise(row_len, 0x1010)
    got = d(g0)
    ops.mul_add(field, got, coeffs[1], d(s0))
    want = g0.copy()
    orc.mul_add(field.ID, want, coeffs[1], s0)
    assert np.array_equal(h(got), want)
    into = d(np.zeros(row_len, np.uint8))
    ops.mul_into(field, into, coeffs[2], d(s0))
    assign = d(s0)
    ops.mul_assign(field, assign, coeffs[2])
    assert np.array_equal(h(into), h(assign))
    sc0 = noise(row_len * len(coeffs), 0x2020)
    sc = d(sc0)
    ops.mul_add_scatter(field, sc, row_len, coeffs, d(s0))
    want = sc0.copy()
    orc.mul_add_scatter(field.ID, want, row_len, coeffs, s0)
    assert np.array_equal(h(sc), want)
    rev = [coeffs[2], coeffs[1], coeffs[0]]
    mx0 = noise(row_len * 3, 0x4040)
    mx = d(mx0)
    ops.mul_add_matrix(field, mx, row_len, 3, [(coeffs[:3], d(s0)), (rev, d(s1))])
    want = mx0.copy()
    orc.mul_add_matrix(field.ID, want, row_len, 3, coeffs[:3] + rev, [s0, s1])
    assert np.array_equal(h(mx), want)


def test_gf8d_prepared_all_coefficients(cuda):
    # tests/ops.rs:1168-1181
    src = noise(64, 0x11D5)
    for c in (0, 1, 2, 0x53, 0xFF):
        p = ops.Coeff(Gf8D, c)
        assert p.value() == c
        g0 = noise(64, 0x11D6)
        a, b = d(g0), d(g0)
        ops.mul_add_with(a, p, d(src))
        ops.mul_add(Gf8D, b, c, d(src))
        assert np.array_equal(h(a), h(b))


# ---------------------------------------------------------------- device-specific edges

@pytest.mark.parametrize("field", [Gf8D, Gf16, Gf32])
def test_unaligned_and_mixed_alignment_buffers(cuda, field):
    """Pointers at every offset mod 16 (shared or mixed) take the scalar or
    vector path; both must agree with the oracle."""
    b = field.BYTES
    k, m = 5, 3
    pool = d(noise(1 << 16, 0xA11))
    host = h(pool)
    rl = 16 * 37 * b + 6 * b
    for shared in (0, b, 4 * b if 4 * b < 16 else b, 16 - b):
        for mixed in (False, True):
            soff = [1024 * (t + 1) + (shared if not mixed else (shared + t * b) % 16) for t in range(k)]
            doff = 40000 + shared
            coeffs = read(field, noise(k * m * b, 0xC0 + shared))
            srcs = [pool[o:o + rl] for o in soff]
            out = pool[doff:doff + m * rl]
            before = h(out).copy()
            ops.mul_add_matrix(field, out, rl, m, [(coeffs[t * m:(t + 1) * m], srcs[t]) for t in range(k)])
            want = before.copy()
            orc.mul_add_matrix(field.ID, want, rl, m, coeffs, [host[o:o + rl].copy() for o in soff])
            assert np.array_equal(h(out), want), (shared, mixed)
            pool[doff:doff + m * rl] = torch.from_numpy(before).cuda()


@pytest.mark.parametrize("field,k,m", [(Gf8B, 64, 16), (Gf8D, 60, 3), (Gf16, 32, 8), (Gf32, 16, 4),
                                       (Gf8D, 3, 33), (Gf16, 40, 1)])
def test_large_k_m_tiling(cuda, field, k, m):
    """Many sources (chunked into several launches) and many rows (several
    row passes) agree with the oracle, overwrite and accumulate."""
    b = field.BYTES
    rl = 4096 + 48 * b
    sources = [noise(rl, 0x900 + t) for t in range(k)]
    coeffs = read(field, noise(k * m * b, 0x9A0 + k))
    want = np.zeros(rl * m, np.uint8)
    orc.dot_product_matrix(field.ID, want, rl, m, coeffs, sources)
    ds = [d(s) for s in sources]
    got = d(noise(rl * m, 0x9B0))
    plan = ops.Plan.matrix(field, k, m, coeffs)
    ops.dot_product_matrix_with(got, rl, m, plan, ds)
    assert np.array_equal(h(got), want)
    got2 = d(noise(rl * m, 0x9B0))
    ops.dot_product_matrix(field, got2, rl, m, [(coeffs[t * m:(t + 1) * m], ds[t]) for t in range(k)])
    assert np.array_equal(h(got2), want)
    acc0 = noise(rl * m, 0x9C0)
    acc = d(acc0)
    ops.mul_add_matrix_with(acc, rl, m, plan, ds)
    assert np.array_equal(h(acc), want ^ acc0)


@pytest.mark.parametrize("field,k,m,ovr", [(Gf8D, 10, 4, True), (Gf8B, 1, 1, False), (Gf8D, 14, 3, True),
                                           (Gf8D, 6, 2, False), (Gf8B, 7, 4, False), (Gf8D, 11, 4, True)])
def test_byte_table_kernel_at_4mib(cuda, field, k, m, ovr):
    """Rows of 4 MiB and more take the byte-table kernel (one lookup per
    source byte); check it bit-exact, with an unaligned tail."""
    rl = (4 << 20) + 16 + 5
    sources = [noise(rl, 0xB00 + t) for t in range(k)]
    coeffs = read(field, noise(k * m, 0xB80 + k))
    init = noise(rl * m, 0xBC0)
    want = init.copy()
    if ovr:
        orc.dot_product_matrix(field.ID, want, rl, m, coeffs, sources)
    else:
        orc.mul_add_matrix(field.ID, want, rl, m, coeffs, sources)
    got = d(init)
    plan = ops.Plan.matrix(field, k, m, coeffs)
    ds = [d(s) for s in sources]
    if ovr:
        ops.dot_product_matrix_with(got, rl, m, plan, ds)
    else:
        ops.mul_add_matrix_with(got, rl, m, plan, ds)
    g = h(got)
    assert np.array_equal(g, want)
