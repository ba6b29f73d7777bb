"""Field markers and host scalar arithmetic for the fields of the hot path.

Mirrors the reference's `Field` types (src/field/mod.rs:110-144): each marker
carries `ID` (the fgfc_field code), `NAME`, `BYTES` and scalar `mul`, `inv`,
`div`, `pow`. The scalar arithmetic is used on the host to build coding and
decode matrices (RS recipes below); vector work goes to the device.

  Gf8B: GF(2)[x]/(x^8+x^4+x^3+x+1), generator 0x03       (src/field/gf8b.rs:57)
  Gf8D: GF(2)[x]/(x^8+x^4+x^3+x^2+1), generator 0x02     (src/field/gf8d.rs:40)
  Gf16: Gf8B[u]/(u^2+u+0x20), bytes [a, b] for a + b*u   (src/field/gf16.rs:54-60)
  Gf32: Gf16[v]/(v^2+v+0x2000), little-endian halves     (src/field/gf32.rs:36-42)
  Gf64: Gf32[w]/(w^2+w+0x20000000), little-endian halves (src/field/gf64.rs:1-11)
  FanPaar8/16/32/64: the canonical Fan-Paar tower        (src/field/fan_paar.rs)
inv(0) = 0 and x/0 = 0 (src/field/mod.rs:38-41).
"""
from __future__ import annotations


def _log_tables(low: int, gen: int) -> tuple[list[int], list[int]]:
    exp = [0] * 512
    log = [0] * 256
    v = 1
    for i in range(255):
        exp[i] = v
        a, acc = v, 0
        for b in range(8):
            if (gen >> b) & 1:
                acc ^= a
            a = ((a << 1) & 0xFF) ^ (low if a & 0x80 else 0)
        v = acc
    for i in range(255, 512):
        exp[i] = exp[i - 255]
    for i in range(255):
        log[exp[i]] = i
    return exp, log


class _Flat8:
    ID = -1
    NAME = ""
    BYTES = 1
    BITS = 8
    POLY = 0
    GENERATOR = 0
    _exp: list[int]
    _log: list[int]

    @classmethod
    def mul(cls, a: int, b: int) -> int:
        if a == 0 or b == 0:
            return 0
        return cls._exp[cls._log[a] + cls._log[b]]

    @classmethod
    def inv(cls, a: int) -> int:
        return 0 if a == 0 else cls._exp[255 - cls._log[a]]


class Gf8B(_Flat8):
    ID = 0
    NAME = "GF(2^8)"
    POLY = 0x11B
    GENERATOR = 0x03
    _exp, _log = _log_tables(0x1B, 0x03)


class Gf8D(_Flat8):
    ID = 1
    NAME = "GF(2^8)/0x11D"
    POLY = 0x11D
    GENERATOR = 0x02
    _exp, _log = _log_tables(0x1D, 0x02)


class Gf16:
    ID = 2
    NAME = "GF(2^16)"
    BYTES = 2
    BITS = 16
    DELTA = 0x20
    GENERATOR = 0x0108

    @staticmethod
    def mul(x: int, y: int) -> int:
        a, b, c, d = x & 0xFF, x >> 8, y & 0xFF, y >> 8
        m = Gf8B.mul
        ac, bd = m(a, c), m(b, d)
        return (ac ^ m(0x20, bd)) | ((m(a ^ b, c ^ d) ^ ac) << 8)

    @staticmethod
    def inv(x: int) -> int:
        if x == 0:
            return 0
        a, b = x & 0xFF, x >> 8
        m = Gf8B.mul
        norm = m(a, a) ^ m(a, b) ^ m(0x20, m(b, b))
        ni = Gf8B.inv(norm)
        return m(a ^ b, ni) | (m(b, ni) << 8)


class Gf32:
    ID = 3
    NAME = "GF(2^32)"
    BYTES = 4
    BITS = 32
    DELTA = 0x2000
    GENERATOR = 0x0001_0002

    @staticmethod
    def mul(x: int, y: int) -> int:
        a, b, c, d = x & 0xFFFF, x >> 16, y & 0xFFFF, y >> 16
        m = Gf16.mul
        ac, bd = m(a, c), m(b, d)
        return (ac ^ m(0x2000, bd)) | ((m(a ^ b, c ^ d) ^ ac) << 16)

    @staticmethod
    def inv(x: int) -> int:
        if x == 0:
            return 0
        a, b = x & 0xFFFF, x >> 16
        m = Gf16.mul
        norm = m(a, a) ^ m(a, b) ^ m(0x2000, m(b, b))
        ni = Gf16.inv(norm)
        return m(a ^ b, ni) | (m(b, ni) << 16)


def _fp_low(bits: int) -> int:
    return (1 << bits) - 1


def _fp_mul_alpha(v: int, bits: int) -> int:
    """Multiply by a level's top tower generator (src/field/fan_paar.rs:67-76)."""
    if bits == 1:
        return v & 1
    h = bits // 2
    a0, a1 = v & _fp_low(h), v >> h
    return a1 | ((a0 ^ _fp_mul_alpha(a1, h)) << h)


def _fp_mul(x: int, y: int, bits: int) -> int:
    """Karatsuba product of the tower X^2 + alpha X + 1 (fan_paar.rs:80-94)."""
    if bits == 1:
        return x & y & 1
    h = bits // 2
    m = _fp_low(h)
    a0, a1, b0, b1 = x & m, x >> h, y & m, y >> h
    z0, z2 = _fp_mul(a0, b0, h), _fp_mul(a1, b1, h)
    z1 = _fp_mul(a0 ^ a1, b0 ^ b1, h) ^ z0 ^ z2
    return (z0 ^ z2) | ((z1 ^ _fp_mul_alpha(z2, h)) << h)


def _fp_inv(x: int, bits: int) -> int:
    """Conjugate times inverse norm, inv(0) = 0 (fan_paar.rs:137-148)."""
    if bits == 1:
        return x & 1
    h = bits // 2
    a0, a1 = x & _fp_low(h), x >> h
    a0z1 = a0 ^ _fp_mul_alpha(a1, h)
    norm = _fp_mul(a0, a0z1, h) ^ _fp_mul(a1, a1, h)
    ni = _fp_inv(norm, h)
    return _fp_mul(ni, a0z1, h) | (_fp_mul(ni, a1, h) << h)


class _FanPaar:
    """Canonical Fan-Paar binary tower (src/field/fan_paar.rs:1-14): each
    level of 2h bits is h-bit[X]/(X^2 + alpha X + 1), alpha the h-bit level's
    own top generator; an element is lo + hi*X, lo in the low h bits."""
    ID = -1
    NAME = ""
    BYTES = 1
    BITS = 8
    GENERATOR = 0

    @classmethod
    def mul(cls, a: int, b: int) -> int:
        return _fp_mul(a & _fp_low(cls.BITS), b & _fp_low(cls.BITS), cls.BITS)

    @classmethod
    def inv(cls, a: int) -> int:
        return _fp_inv(a & _fp_low(cls.BITS), cls.BITS)


class FanPaar8(_FanPaar):
    ID = 4
    NAME = "Fan-Paar GF(2^8)"
    BYTES, BITS = 1, 8
    GENERATOR = 0x2D  # src/field/fan_paar.rs:537-548


class FanPaar16(_FanPaar):
    ID = 5
    NAME = "Fan-Paar GF(2^16)"
    BYTES, BITS = 2, 16
    GENERATOR = 0xE2DE  # fan_paar.rs:549-562


class FanPaar32(_FanPaar):
    ID = 6
    NAME = "Fan-Paar GF(2^32)"
    BYTES, BITS = 4, 32
    GENERATOR = 0x03E2_1CEA  # fan_paar.rs:563-576


class FanPaar64(_FanPaar):
    ID = 8
    NAME = "Fan-Paar GF(2^64)"
    BYTES, BITS = 8, 64
    GENERATOR = 0x070F_870D_CD9C_1D88  # fan_paar.rs:577-590


class Gf64:
    """GF(2^64) = Gf32[w]/(w^2 + w + 0x20000000), a + b*w with a in the low
    half (src/field/gf64.rs:1-11,120-151)."""
    ID = 7
    NAME = "GF(2^64)"
    BYTES = 8
    BITS = 64
    DELTA = 0x2000_0000
    GENERATOR = 0x0000_0001_0000_0004

    @staticmethod
    def mul(x: int, y: int) -> int:
        a, b, c, d = x & 0xFFFFFFFF, x >> 32, y & 0xFFFFFFFF, y >> 32
        m = Gf32.mul
        ac, bd = m(a, c), m(b, d)
        return (ac ^ m(0x2000_0000, bd)) | ((m(a ^ b, c ^ d) ^ ac) << 32)

    @staticmethod
    def inv(x: int) -> int:
        if x == 0:
            return 0
        a, b = x & 0xFFFFFFFF, x >> 32
        m = Gf32.mul
        norm = m(a, a) ^ m(a, b) ^ m(0x2000_0000, m(b, b))
        ni = Gf32.inv(norm)
        return m(a ^ b, ni) | (m(b, ni) << 32)


FIELDS = {f.ID: f for f in (Gf8B, Gf8D, Gf16, Gf32, FanPaar8, FanPaar16, FanPaar32, Gf64, FanPaar64)}


def div(field, a: int, b: int) -> int:
    return 0 if a == 0 or b == 0 else field.mul(a, field.inv(b))


def pow_(field, a: int, e: int) -> int:
    r, base = 1, a
    while e:
        if e & 1:
            r = field.mul(r, base)
        base = field.mul(base, base)
        e >>= 1
    return r


# ---------------------------------------------------------------- RS recipes
# The reference leaves coding-matrix construction to its callers
# (src/lib.rs:115-116). These are the recipes the encode/reconstruct paths use.

def cauchy(field, m: int, k: int, x0: int | None = None) -> list[list[int]]:
    """c[i][j] = inv(x_i + y_j), x_i = x0 + i (default x0 = k), y_j = j."""
    x0 = k if x0 is None else x0
    return [[field.inv((x0 + i) ^ j) for j in range(k)] for i in range(m)]


def encode_plan_coeffs(c: list[list[int]]) -> tuple[int, int, list[int]]:
    """Transpose an m x k parity matrix into Plan::matrix(k, m) order
    (one plan row per source term, src/ops.rs:712-718)."""
    m, k = len(c), len(c[0]) if c else 0
    return k, m, [c[i][t] for t in range(k) for i in range(m)]


def invert(field, a: list[list[int]]) -> list[list[int]]:
    """Gauss-Jordan inverse over the field; raises ValueError if singular."""
    n = len(a)
    aug = [list(row) + [1 if i == j else 0 for j in range(n)] for i, row in enumerate(a)]
    for col in range(n):
        piv = next((r for r in range(col, n) if aug[r][col]), None)
        if piv is None:
            raise ValueError("singular matrix")
        aug[col], aug[piv] = aug[piv], aug[col]
        pinv = field.inv(aug[col][col])
        aug[col] = [field.mul(v, pinv) for v in aug[col]]
        for r in range(n):
            if r != col and aug[r][col]:
                f = aug[r][col]
                aug[r] = [v ^ field.mul(f, w) for v, w in zip(aug[r], aug[col])]
    return [row[n:] for row in aug]


def decode_rows(field, c: list[list[int]], survivors: list[int], erased: list[int]) -> list[list[int]]:
    """Rows D (len(erased) x k) with codeword[e] = sum_t D[e][t] * codeword[survivors[t]]
    for the systematic generator [I_k ; C]."""
    m, k = len(c), len(c[0])

    def gen(r: int, col: int) -> int:
        return (1 if r == col else 0) if r < k else c[r - k][col]

    sub = [[gen(s, j) for j in range(k)] for s in survivors]
    inv = invert(field, sub)
    out = []
    for e in erased:
        row = []
        for t in range(k):
            acc = 0
            for q in range(k):
                acc ^= field.mul(gen(e, q), inv[q][t])
            row.append(acc)
        out.append(row)
    return out
