"""Coding and decode matrices through the C ABI (decode.cpp), host only.

Pinned to the oracle's Gauss-Jordan restatement (oracle/fgf_oracle.c,
orc_decode_matrix) for every one of the C(14,4) = 1001 erasure patterns of
the RS(10,4) Gf8D Cauchy code, for the tower fields, and to the reference's
own round-trip recipe (tests/ops.rs:897-950: parity g^((i+1)(j+1)) over
Gf8B, data rows 1 and 4 lost)."""
from itertools import combinations

import numpy as np
import pytest

from fgf_b200 import codes
from fgf_b200._lib import FgfError
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32, cauchy, pow_
from oracle import orc


def test_cauchy_matches_the_recipe():
    for field, m, k in ((Gf8D, 4, 10), (Gf16, 8, 32), (Gf32, 4, 16), (Gf8B, 16, 64)):
        assert codes.cauchy_matrix(field, m, k) == cauchy(field, m, k)
        assert codes.cauchy_matrix(field, m, k) == orc.cauchy(field.ID, m, k).tolist()


def test_every_rs10_4_erasure_pattern_matches_the_oracle():
    k, m = 10, 4
    c = codes.cauchy_matrix(Gf8D, m, k)
    carr = np.array(c, dtype=np.uint32)
    n = 0
    for erased in combinations(range(k + m), m):
        survivors = [i for i in range(k + m) if i not in erased][:k]
        got = codes.decode_matrix(Gf8D, c, survivors, list(erased))
        want = orc.decode_matrix(Gf8D.ID, carr, survivors, list(erased))  # rows: erased x k
        assert got == [int(want[e][t]) for t in range(k) for e in range(m)], erased
        n += 1
    assert n == 1001


@pytest.mark.parametrize("field,k,m", [(Gf16, 32, 8), (Gf32, 16, 4), (Gf8B, 64, 16)],
                         ids=["gf16", "gf32", "gf8b"])
def test_tower_and_large_codes(field, k, m):
    c = codes.cauchy_matrix(field, m, k)
    rng = np.random.default_rng(field.ID)
    erased = sorted(int(x) for x in rng.choice(k + m, size=m, replace=False))
    survivors = [i for i in range(k + m) if i not in erased]
    got = codes.decode_matrix(field, c, survivors, erased)
    want = orc.decode_matrix(field.ID, np.array(c, dtype=np.uint32), survivors, erased)
    assert got == [int(want[e][t]) for t in range(k) for e in range(m)]


def test_reference_round_trip_recipe():
    """tests/ops.rs:897-950: k = 6, m = 3, coeff(i, j) = g^((i+1)(j+1)) in Gf8B;
    data rows 1 and 4 are rebuilt from the other data rows and parity rows 0, 1."""
    k, m = 6, 3
    parity = [[pow_(Gf8B, Gf8B.GENERATOR, (i + 1) * (j + 1)) for i in range(k)] for j in range(m)]
    survivors = [0, 2, 3, 5, k + 0, k + 1]
    d = codes.decode_matrix(Gf8B, parity, survivors, [1, 4])
    data = [orc.noise(64, 0x5150 + i) for i in range(k)]
    shards = data + [np.zeros(64, np.uint8) for _ in range(m)]
    for j in range(m):
        orc.dot_product(Gf8B.ID, shards[k + j], [parity[j][i] for i in range(k)], data)
    for e, lost in enumerate([1, 4]):
        out = np.zeros(64, np.uint8)
        orc.dot_product(Gf8B.ID, out, [d[t * 2 + e] for t in range(k)], [shards[s] for s in survivors])
        assert np.array_equal(out, data[lost])


def test_singular_and_bad_indices_are_rejected():
    c = [[1, 1], [1, 1]]  # two identical parity rows: {parity 0, parity 1} cannot rebuild 2 data shards
    with pytest.raises(FgfError, match="singular"):
        codes.decode_matrix(Gf8D, c, [2, 3], [0, 1])
    with pytest.raises(FgfError, match="repeated"):
        codes.decode_matrix(Gf8D, c, [0, 0], [1])
    with pytest.raises(FgfError, match="out of range"):
        codes.decode_matrix(Gf8D, c, [0, 1], [7])
    with pytest.raises(FgfError, match="nonzero"):
        codes.cauchy_matrix(Gf8D, 2, 3, 1)  # x_1 = 2 = y_2
