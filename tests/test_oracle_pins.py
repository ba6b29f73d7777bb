"""Pin the oracle (and the product's host arithmetic) to every known answer
in the reference's own tests, doctests and table self-tests.

The reference (Rust) cannot be built here, so these known answers are the
parity anchor; tests/golden/known_answers.json holds them with citations.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import orc
from fgf_b200 import fields

GOLD = json.loads((Path(__file__).parent / "golden" / "known_answers.json").read_text())
F = {"gf8b": orc.GF8B, "gf8d": orc.GF8D, "gf16": orc.GF16, "gf32": orc.GF32}
HOST = {"gf8b": fields.Gf8B, "gf8d": fields.Gf8D, "gf16": fields.Gf16, "gf32": fields.Gf32}


@pytest.mark.parametrize("case", GOLD["products"], ids=lambda c: f"{c['field']}-{c['a']}x{c['b']}")
def test_known_answer_products(case):
    f = F[case["field"]]
    a, b, want = (int(case[k], 16) for k in ("a", "b", "product"))
    assert orc.mul(f, a, b) == want
    assert orc.mul(f, b, a) == want
    assert HOST[case["field"]].mul(a, b) == want


@pytest.mark.parametrize("case", GOLD["mul_add_vectors"], ids=lambda c: c["source"])
def test_doctest_mul_add_vectors(case):
    f = F[case["field"]]
    src = np.frombuffer(bytes.fromhex(case["src"]), dtype=np.uint8).copy()
    dst = np.frombuffer(bytes.fromhex(case["dst"]), dtype=np.uint8).copy()
    orc.mul_add(f, dst, int(case["coeff"], 16), src)
    assert dst.tobytes().hex() == case["want"]
    # src/lib.rs:47-49: applying the same term twice cancels it
    orc.mul_add(f, dst, int(case["coeff"], 16), src)
    assert dst.tobytes().hex() == case["dst"]


def test_gf8_xtime_and_log_products_agree_exhaustively():
    # tests/algebra.rs: table product == shift/XOR product for all 65536 pairs
    for f in (orc.GF8B, orc.GF8D):
        for a in range(256):
            for b in range(0, 256, 1):
                assert orc.mul(f, a, b) == orc.mul_xtime(f, a, b)


def test_fields_differ_on_63232_products():
    # tests/algebra.rs:233-248
    differ = sum(1 for a in range(256) for b in range(256)
                 if orc.mul(orc.GF8B, a, b) != orc.mul(orc.GF8D, a, b))
    assert differ == GOLD["gf8b_gf8d_differing_products"]


@pytest.mark.parametrize("f", [orc.GF8B, orc.GF8D])
def test_gf8_inverse_laws(f):
    # tests/algebra.rs:58-66,147-155: inv(0) = 0, inverse backends agree
    assert orc.inv(f, 0) == 0 and orc.div(f, 0x57, 0) == 0
    for a in range(1, 256):
        assert orc.inv(f, a) == orc.inv_xtime(f, a)
        assert orc.mul(f, a, orc.inv(f, a)) == 1
        assert orc.div(f, a, a) == 1


@pytest.mark.parametrize("name", ["gf8b", "gf8d", "gf16", "gf32"])
def test_generator_orders(name):
    # gf8d.rs:17-19, gf16.rs:43, algebra.rs:457-465
    case = GOLD["generators"][name]
    f, g, order = F[name], int(case["generator"], 16), case["order"]
    assert orc.pow_(f, g, order) == 1
    for factor in case["prime_factors"]:
        assert orc.pow_(f, g, order // factor) != 1


def _sample16():
    vals = [0, 1, 0x0100, 0x00FF, 0xFF00, 0xFFFF, 0x0108, 0x1234, 0xBEEF]
    return vals + [int(x) for x in orc.noise(64, 0x1616).view(np.uint16)]


def test_gf16_karatsuba_matches_schoolbook():
    # tests/algebra.rs:257-278: schoolbook (a+bu)(c+du) with u^2 = u + DELTA
    m = lambda x, y: orc.mul_xtime(orc.GF8B, x, y)  # noqa: E731
    for x in _sample16():
        for y in _sample16():
            a, b, c, d = x & 0xFF, x >> 8, y & 0xFF, y >> 8
            ac, ad, bc, bd = m(a, c), m(a, d), m(b, c), m(b, d)
            want = (ac ^ m(0x20, bd)) | ((ad ^ bc ^ bd) << 8)
            assert orc.mul(orc.GF16, x, y) == want
            assert fields.Gf16.mul(x, y) == want


def test_gf16_inverse_and_embedding():
    for x in _sample16():
        if x:
            assert orc.mul(orc.GF16, x, orc.inv(orc.GF16, x)) == 1
            assert fields.Gf16.inv(x) == orc.inv(orc.GF16, x)
    assert orc.inv(orc.GF16, 0) == 0
    # tests/algebra.rs:336-357: elements with zero extension multiply as in Gf8B
    for a in range(0, 256, 5):
        for b in range(0, 256, 7):
            assert orc.mul(orc.GF16, a, b) == orc.mul(orc.GF8B, a, b)


def test_gf32_tower_matches_schoolbook():
    # tests/algebra.rs:402-436
    vals = [0, 1, 0x0000FFFF, 0xFFFF0000, 0xDEADBEEF, 0x56781234]
    vals += [int(x) for x in orc.noise(96, 0x3232).view(np.uint32)]
    m16 = lambda x, y: orc.mul(orc.GF16, x, y)  # noqa: E731
    for x in vals:
        for y in vals:
            a, b, c, d = x & 0xFFFF, x >> 16, y & 0xFFFF, y >> 16
            want = (m16(a, c) ^ m16(0x2000, m16(b, d))) | ((m16(a, d) ^ m16(b, c) ^ m16(b, d)) << 16)
            assert orc.mul(orc.GF32, x, y) == want
            assert fields.Gf32.mul(x, y) == want
        if x:
            assert orc.mul(orc.GF32, x, orc.inv(orc.GF32, x)) == 1
    # src/field/gf32.rs:13-29 doctest: X * inv(X) == 1 for X = 0x5678_1234
    assert orc.mul(orc.GF32, 0x56781234, orc.inv(orc.GF32, 0x56781234)) == 1


def test_nibble_split_reconstructs_products():
    # src/kernel/tables.rs:511-521: lo[x & 15] ^ hi[x >> 4] == c * x
    for f in (orc.GF8B, orc.GF8D):
        for c in range(256):
            lo = [orc.mul(f, c, n) for n in range(16)]
            hi = [orc.mul(f, c, n << 4) for n in range(16)]
            for x in range(256):
                assert lo[x & 15] ^ hi[x >> 4] == orc.mul(f, c, x)


def test_tower_byte_factors_reconstruct_products():
    # src/kernel/tables.rs:556-575: even = f0*a ^ f2*b, odd = f1*b ^ f3*a,
    # with f0 = c0, f1 = c0 ^ c1, f2 = 0x20*c1, f3 = c1 over Gf8B.
    m = lambda x, y: orc.mul(orc.GF8B, x, y)  # noqa: E731
    for coeff in (0, 1, 0x0108, 0x2000, 0xFFFF, 0x1234):
        c0, c1 = coeff & 0xFF, coeff >> 8
        for value in (0, 1, 0x00FF, 0xFF00, 0xBEEF):
            a, b = value & 0xFF, value >> 8
            even = m(c0, a) ^ m(m(0x20, c1), b)
            odd = m(c0 ^ c1, b) ^ m(c1, a)
            assert even | (odd << 8) == orc.mul(orc.GF16, value, coeff)


def test_noise_stream_matches_reference_lcg():
    # tests/ops.rs:17-27, restated in Python as an independent check
    def noise(n, seed):
        s = (seed | 1) & (2 ** 64 - 1)
        out = []
        for _ in range(n):
            s = (s * 6364136223846793005 + 1) & (2 ** 64 - 1)
            out.append((s >> 33) & 0xFF)
        return bytes(out)

    for seed in (0, 1, 0xA1, 0x7A2, 0x5150):
        assert orc.noise(257, seed).tobytes() == noise(257, seed)


def test_erasure_round_trip_oracle():
    # tests/ops.rs:897-950 (Cramer) generalised: Gauss-Jordan decode rows
    # recover erased rows from any k survivors of [I ; C].
    k, m, L = 6, 3, 1024
    for f in (orc.GF8B, orc.GF8D, orc.GF16):
        c = orc.cauchy(f, m, k)
        data = [orc.noise(L, 0x5150 + i) for i in range(k)]
        parity = np.zeros(m * L, dtype=np.uint8)
        orc.dot_product_matrix(f, parity, L, m, [c[i][t] for t in range(k) for i in range(m)], data)
        code = data + [parity[i * L:(i + 1) * L].copy() for i in range(m)]
        erased = [1, 4, 7]
        survivors = [i for i in range(k + m) if i not in erased][:k]
        d = orc.decode_matrix(f, c, survivors, erased)
        hostd = fields.decode_rows(fields.FIELDS[f], c.tolist(), survivors, erased)
        assert d.tolist() == hostd
        out = np.zeros(len(erased) * L, dtype=np.uint8)
        orc.dot_product_matrix(f, out, L, len(erased),
                               [d[j][t] for t in range(k) for j in range(len(erased))],
                               [code[s] for s in survivors])
        for j, e in enumerate(erased):
            assert np.array_equal(out[j * L:(j + 1) * L], code[e])


def test_host_cauchy_matches_oracle():
    for f, fh in ((orc.GF8D, fields.Gf8D), (orc.GF8B, fields.Gf8B), (orc.GF16, fields.Gf16)):
        assert orc.cauchy(f, 4, 10).tolist() == fields.cauchy(fh, 4, 10)


# ---------------------------------------------------------------- Fan-Paar towers
FP = GOLD["fan_paar"]
FPF = {"fp8": (orc.FP8, fields.FanPaar8), "fp16": (orc.FP16, fields.FanPaar16), "fp32": (orc.FP32, fields.FanPaar32)}


@pytest.mark.parametrize("case", FP["products"], ids=lambda c: f"{c['field']}-{c['a']}x{c['b']}")
def test_fan_paar_known_products(case):
    # tests/algebra.rs:478-495
    f, host = FPF[case["field"]]
    a, b, want = (int(case[k], 16) for k in ("a", "b", "product"))
    assert orc.mul(f, a, b) == want and orc.mul(f, b, a) == want
    assert host.mul(a, b) == want


def test_fan_paar_known_squares():
    for case in FP["squares"]:
        f, host = FPF[case["field"]]
        a, want = int(case["a"], 16), int(case["square"], 16)
        assert orc.mul(f, a, a) == want and host.mul(a, a) == want


@pytest.mark.parametrize("name", ["fp8", "fp16", "fp32"])
def test_fan_paar_round_trips(name):
    # tests/algebra.rs:499-524: a * inv(a) == 1 on the listed values (the
    # squares agree with products by construction here: one multiply)
    f, host = FPF[name]
    for v in FP["round_trip_values"][name]:
        a = int(v, 16)
        assert host.mul(a, a) == orc.mul(f, a, a)
        if a:
            assert orc.mul(f, a, orc.inv(f, a)) == 1
            assert host.mul(a, host.inv(a)) == 1
    assert orc.inv(f, 0) == 0 and host.inv(0) == 0


@pytest.mark.parametrize("case", FP["generators"], ids=lambda c: c["field"])
def test_fan_paar_generators_have_full_order(case):
    # tests/algebra.rs:527-552
    f, host = FPF[case["field"]]
    g, order = int(case["generator"], 16), case["order"]
    assert host.GENERATOR == g
    assert orc.pow_(f, g, order) == 1
    for q in case["factors"]:
        assert orc.pow_(f, g, order // q) != 1


def test_fan_paar_byte_products_nest():
    # tests/algebra.rs:555-576: a byte keeps its products in the wider levels
    for a, b in FP["nested_byte_products"]["pairs"]:
        a, b = int(a, 16), int(b, 16)
        p = orc.mul(orc.FP8, a, b)
        assert orc.mul(orc.FP16, a, b) == p and orc.mul(orc.FP32, a, b) == p


def test_fan_paar_names():
    for name, (_, host) in FPF.items():
        assert host.NAME == FP["names"][name]


# ---------------------------------------------------------------- 8-byte fields
WIDE = GOLD["wide_fields"]


def test_gf64_schoolbook_inverse_and_order():
    # tests/algebra.rs:412-420,439-471
    vals = [int(v, 16) for v in WIDE["gf64_sample"]["values"]]
    delta = int(WIDE["gf64_sample"]["delta"], 16)

    def school(x, y):
        a, b, c, d = x & 0xFFFFFFFF, x >> 32, y & 0xFFFFFFFF, y >> 32
        m = lambda u, v: orc.mul(orc.GF32, u, v)  # noqa: E731
        return (m(a, c) ^ m(delta, m(b, d))) | ((m(a, d) ^ m(b, c) ^ m(b, d)) << 32)

    for i, a in enumerate(vals):
        b = vals[(i * 7 + 3) % len(vals)]
        assert orc.mul64(orc.GF64, a, b) == school(a, b) == fields.Gf64.mul(a, b)
        if a:
            assert orc.mul64(orc.GF64, a, orc.inv64(orc.GF64, a)) == 1
            assert fields.Gf64.mul(a, fields.Gf64.inv(a)) == 1
    g = int(WIDE["gf64_generator"]["generator"], 16)
    assert fields.Gf64.GENERATOR == g
    assert orc.pow64(orc.GF64, g, (1 << 64) - 1) == 1
    for q in WIDE["gf64_generator"]["factors"]:
        assert orc.pow64(orc.GF64, g, ((1 << 64) - 1) // q) != 1


def test_fan_paar_64_vectors():
    # tests/algebra.rs:491-494,517-523,547-551,555-576
    for case in WIDE["fp64_products"]:
        a, b, want = (int(case[k], 16) for k in ("a", "b", "product"))
        assert orc.mul64(orc.FP64, a, b) == want == fields.FanPaar64.mul(a, b)
    for v in WIDE["fp64_round_trip_values"]["values"]:
        a = int(v, 16)
        if a:
            assert orc.mul64(orc.FP64, a, orc.inv64(orc.FP64, a)) == 1
            assert fields.FanPaar64.mul(a, fields.FanPaar64.inv(a)) == 1
    g = int(WIDE["fp64_generator"]["generator"], 16)
    assert fields.FanPaar64.GENERATOR == g
    assert orc.pow64(orc.FP64, g, (1 << 64) - 1) == 1
    for q in WIDE["fp64_generator"]["factors"]:
        assert orc.pow64(orc.FP64, g, ((1 << 64) - 1) // q) != 1
    for a, b in FP["nested_byte_products"]["pairs"]:
        a, b = int(a, 16), int(b, 16)
        assert orc.mul64(orc.FP64, a, b) == orc.mul(orc.FP8, a, b)


def test_wide_field_names():
    assert fields.Gf64.NAME == WIDE["names"]["gf64"] and fields.FanPaar64.NAME == WIDE["names"]["fp64"]


@pytest.mark.parametrize("fid", [orc.GF64, orc.FP64])
def test_wide_oracle_ops_agree_with_the_scalar_product(fid):
    """The oracle's vector ops with 64-bit coefficients (including values at
    and above 2^63) equal the scalar product applied element by element."""
    ln, m = 8 * 40, 3
    c = [0x8000000100000003, 5, 0xFFFFFFFFFFFFFFFF]
    src = orc.noise(ln, 1)
    rows = orc.noise(m * ln, 2)
    want = rows.copy().view("<u8")
    x = src.view("<u8")
    for j in range(m):
        for i in range(ln // 8):
            want[j * (ln // 8) + i] ^= np.uint64(orc.mul64(fid, c[j], int(x[i])))
    got = rows.copy()
    orc.mul_add_scatter(fid, got, ln, c, src)
    assert np.array_equal(got.view("<u8"), want)
    srcs = [orc.noise(ln, 10 + t) for t in range(m)]
    got = np.zeros(ln, np.uint8)
    orc.dot_product(fid, got, c, srcs)
    want = np.zeros(ln // 8, np.uint64)
    for t in range(m):
        for i, v in enumerate(srcs[t].view("<u8")):
            want[i] ^= np.uint64(orc.mul64(fid, c[t], int(v)))
    assert np.array_equal(got.view("<u8"), want)


def test_gf16_mul_add_doctest():
    """src/lib.rs:53-65: mul_add over Gf16's little-endian bytes equals the
    field product written back as bytes."""
    v = GOLD["gf16_mul_add_doctest"]
    src = np.frombuffer(bytes.fromhex(v["src_le"]), np.uint8).copy()
    dst = np.frombuffer(bytes.fromhex(v["dst0"]), np.uint8).copy()
    coeff = int(v["coeff"], 16)
    orc.mul_add(orc.GF16, dst, coeff, src)
    prod = orc.mul(orc.GF16, int.from_bytes(src.tobytes(), "little"), coeff)
    assert dst.tobytes() == prod.to_bytes(2, "little") == bytes.fromhex(v["product_le"])
