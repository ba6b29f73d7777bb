"""Parity at the workload sizes of the measured configurations, through the C ABI.

The CPU oracle is scalar, so at these sizes it checks element-aligned column
windows (the first and last 4 KiB of every row and six seeded windows in
between): every op of the family is independent column by column, so the
oracle run on the windows of the sources gives exactly the windows of the
result. Full-size properties of the domain cover every byte:

* RS shapes: encode with a systematic code [I; C], erase as many shards as
  there are parity rows, rebuild them from the survivors with the decode
  rows (inverse of the surviving submatrix, inv(0) = 0 convention) and
  compare with the originals, all on the device;
* single-row ops: linearity in the coefficient, (c1 + c2) * s = c1 * s + c2 * s,
  and agreement of the scatter / gather forms with sequences of mul_add.

Shapes (reference ops: src/ops.rs:342-941): Gf16 RS(32,8) on 16 MiB shards,
Gf32 RS(16,4) on 8 MiB, Gf8B RS(64,16) on 4 MiB, Gf8D RS(10,4) reconstruct
on 64 MiB shards, mul_add / mul_add_scatter 1->4 / mul_add_gather 4->1 on
256 MiB buffers with random nonzero coefficients.
"""
import numpy as np
import pytest
import torch

from fgf_b200 import ops
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32, cauchy, decode_rows, encode_plan_coeffs
from oracle import orc

pytestmark = pytest.mark.gpu

WIN = 4096
MIB = 1 << 20


def _windows(n: int, rng) -> list[tuple[int, int]]:
    """Element-aligned windows of a row of n bytes: both ends and six inside."""
    out = [(0, min(WIN, n)), (max(0, n - WIN), n)]
    for _ in range(6):
        a = int(rng.integers(0, max(1, n - WIN))) // 16 * 16
        out.append((a, min(n, a + WIN)))
    return out


def _rand(n: int, gen: torch.Generator) -> torch.Tensor:
    return torch.randint(0, 256, (n,), dtype=torch.uint8, device="cuda", generator=gen)


def _nonzero_coeffs(field, n: int, rng) -> list[int]:
    hi = 1 << (8 * field.BYTES)
    return [int(x) for x in rng.integers(1, hi, size=n, dtype=np.uint64)]


def _systematic(field, k: int, m: int, rng):
    """Random nonzero m x k parity matrix with a set of m erasures (data and
    parity shards mixed) whose surviving k x k submatrix is invertible."""
    for _ in range(50):
        c = [_nonzero_coeffs(field, k, rng) for _ in range(m)]
        erased = sorted(int(x) for x in rng.choice(k + m, size=m, replace=False))
        survivors = [i for i in range(k + m) if i not in erased]
        try:
            d = decode_rows(field, c, survivors, erased)
        except ValueError:
            continue
        return c, erased, survivors, d
    raise AssertionError("no invertible survivor set found")


def _encode_windows_vs_oracle(field, code: torch.Tensor, k: int, m: int, L: int, coeffs: list[int], rng):
    for a, b in _windows(L, rng):
        srcs = [code[t * L + a:t * L + b].cpu().numpy().copy() for t in range(k)]
        want = np.zeros(m * (b - a), np.uint8)
        orc.dot_product_matrix(field.ID, want, b - a, m, coeffs, srcs)
        for j in range(m):
            got = code[(k + j) * L + a:(k + j) * L + b].cpu().numpy()
            assert np.array_equal(got, want[j * (b - a):(j + 1) * (b - a)]), \
                f"parity row {j} window [{a}, {b}) differs from the oracle"


@pytest.mark.parametrize("field,k,m,shard", [
    (Gf16, 32, 8, 16 * MIB),
    (Gf32, 16, 4, 8 * MIB),
    (Gf8B, 64, 16, 4 * MIB),
], ids=["gf16_rs32_8_16MiB", "gf32_rs16_4_8MiB", "gf8b_rs64_16_4MiB"])
def test_tower_and_large_km_encode_and_rebuild(cuda, field, k, m, shard):
    rng = np.random.default_rng(0xC0DE + field.ID)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0xC0DE + field.ID)
    c, erased, survivors, d = _systematic(field, k, m, rng)
    code = torch.empty((k + m) * shard, dtype=torch.uint8, device="cuda")
    code[:k * shard] = _rand(k * shard, gen)
    code[k * shard:] = 0xA5  # overwrite ignores prior contents
    _, _, vals = encode_plan_coeffs(c)
    plan = ops.Plan.matrix(field, k, m, vals)
    shards = [code[i * shard:(i + 1) * shard] for i in range(k + m)]
    ops.dot_product_matrix_with(code[k * shard:], shard, m, plan, shards[:k])
    torch.cuda.synchronize()
    _encode_windows_vs_oracle(field, code, k, m, shard, vals, rng)

    truth = torch.stack([shards[e].clone() for e in erased])
    out = torch.full((m * shard,), 0x3C, dtype=torch.uint8, device="cuda")
    dplan = ops.Plan.matrix(field, k, m, [d[j][t] for t in range(k) for j in range(m)])
    ops.dot_product_matrix_with(out, shard, m, dplan, [shards[s] for s in survivors])
    torch.cuda.synchronize()
    assert torch.equal(out.view(m, shard), truth), "rebuilt shards differ from the originals"


def test_rs10_4_reconstruct_64MiB_shards(cuda):
    k, m, L = 10, 4, 64 * MIB
    rng = np.random.default_rng(0x64)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0x64)
    cm = cauchy(Gf8D, m, k)
    _, _, vals = encode_plan_coeffs(cm)
    code = torch.empty((k + m) * L, dtype=torch.uint8, device="cuda")
    code[:k * L] = _rand(k * L, gen)
    shards = [code[i * L:(i + 1) * L] for i in range(k + m)]
    ops.dot_product_matrix_with(code[k * L:], L, m, ops.Plan.matrix(Gf8D, k, m, vals), shards[:k])
    torch.cuda.synchronize()
    _encode_windows_vs_oracle(Gf8D, code, k, m, L, vals, rng)

    erased = sorted(int(x) for x in rng.choice(k + m, size=m, replace=False))
    survivors = [i for i in range(k + m) if i not in erased][:k]
    truth = {e: shards[e].clone() for e in erased}
    for e in erased:
        shards[e].zero_()  # a real rebuild zeroes the erased rows, then accumulates
    dm = decode_rows(Gf8D, cm, survivors, erased)
    terms = [([dm[j][t] for j in range(m)], shards[s]) for t, s in enumerate(survivors)]
    ops.mul_add_matrix_scattered(Gf8D, code, L, [e * L for e in erased], terms)
    torch.cuda.synchronize()
    for e in erased:
        assert torch.equal(shards[e], truth[e]), f"shard {e} not rebuilt"


@pytest.mark.parametrize("field", [Gf8D, Gf16], ids=lambda f: f.__name__)
def test_mul_add_256MiB(cuda, field):
    n = 256 * MIB
    rng = np.random.default_rng(0xA7 + field.ID)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0xA7 + field.ID)
    c1, c2 = _nonzero_coeffs(field, 2, rng)
    while c2 == c1:
        c2 = _nonzero_coeffs(field, 1, rng)[0]
    src, dst0 = _rand(n, gen), _rand(n, gen)
    dst = dst0.clone()
    ops.mul_add(field, dst, c1, src)
    torch.cuda.synchronize()
    for a, b in _windows(n, rng):
        want = dst0[a:b].cpu().numpy().copy()
        orc.mul_add(field.ID, want, c1, src[a:b].cpu().numpy().copy())
        assert np.array_equal(dst[a:b].cpu().numpy(), want), f"window [{a}, {b}) differs from the oracle"
    ops.mul_add(field, dst, c2, src)           # dst0 + c1 s + c2 s
    other = dst0.clone()
    ops.mul_add(field, other, c1 ^ c2, src)    # dst0 + (c1 + c2) s
    torch.cuda.synchronize()
    assert torch.equal(dst, other), "mul_add is not linear in the coefficient at full size"


def test_mul_add_scatter_and_gather_256MiB(cuda):
    field, n, m = Gf8D, 256 * MIB, 4
    rng = np.random.default_rng(0x5C)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0x5C)
    coeffs = _nonzero_coeffs(field, m, rng)
    src = _rand(n, gen)
    rows0 = _rand(m * n, gen)
    rows = rows0.clone()
    ops.mul_add_scatter(field, rows, n, coeffs, src)
    torch.cuda.synchronize()
    for a, b in _windows(n, rng):
        hs = src[a:b].cpu().numpy().copy()
        for j in range(m):
            want = rows0[j * n + a:j * n + b].cpu().numpy().copy()
            orc.mul_add(field.ID, want, coeffs[j], hs)
            assert np.array_equal(rows[j * n + a:j * n + b].cpu().numpy(), want), \
                f"scatter row {j} window [{a}, {b}) differs from the oracle"
    ref = rows0.clone()
    for j in range(m):
        ops.mul_add(field, ref[j * n:(j + 1) * n], coeffs[j], src)
    torch.cuda.synchronize()
    assert torch.equal(rows, ref), "scatter differs from per-row mul_add at full size"
    del ref, rows0

    srcs = [rows[j * n:(j + 1) * n] for j in range(m)]
    dst0 = _rand(n, gen)
    dst = dst0.clone()
    ops.mul_add_gather(field, dst, coeffs, srcs)
    torch.cuda.synchronize()
    for a, b in _windows(n, rng):
        want = dst0[a:b].cpu().numpy().copy()
        orc.mul_add_gather(field.ID, want, coeffs, [s[a:b].cpu().numpy().copy() for s in srcs])
        assert np.array_equal(dst[a:b].cpu().numpy(), want), f"gather window [{a}, {b}) differs from the oracle"
    ref = dst0.clone()
    for j in range(m):
        ops.mul_add(field, ref, coeffs[j], srcs[j])
    torch.cuda.synchronize()
    assert torch.equal(dst, ref), "gather differs from a sequence of mul_add at full size"
