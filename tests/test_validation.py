"""Geometry validation mirrors the reference's panics (src/ops.rs), message
for message. Every case here is rejected on the host before any device work,
so these run without a GPU; the pointers are never dereferenced."""
import pytest

from fgf_b200 import ops
from fgf_b200.fields import Gf8B, Gf8D, Gf16
from fgf_b200.ops import FgfError

P = 0x7F0000000000  # never dereferenced: every call below fails validation first


def buf(n, off=0):
    return (P + off, n)


def test_dot_product_rejects_mismatched_source_count():
    # tests/ops.rs:952-957
    with pytest.raises(FgfError, match="dot_product: 2 coefficients for 1 sources"):
        ops.dot_product(Gf8B, buf(8), [2, 3], [buf(8, 64)])


def test_dot_product_rejects_wrong_source_length():
    # tests/ops.rs:959-964
    with pytest.raises(FgfError, match="dot_product: source 0 is 7 bytes, expected 8"):
        ops.dot_product(Gf8B, buf(8), [2], [buf(7, 64)])


def test_mul_add_rejects_length_mismatch():
    # tests/ops.rs:970-975
    with pytest.raises(FgfError, match="dst is 8 bytes but src is 4 bytes"):
        ops.mul_add(Gf8B, buf(8), 2, buf(4, 64))


def test_gf16_rejects_odd_length():
    # tests/ops.rs:977-982
    with pytest.raises(FgfError, match="whole number of"):
        ops.mul_add(Gf16, buf(7), 2, buf(7, 64))
    with pytest.raises(FgfError, match=r"mul_add: buffer of 7 bytes is not a whole number of GF\(2\^16\) elements"):
        ops.mul_add(Gf16, buf(7), 2, buf(7, 64))


def test_scatter_rejects_wrong_row_count():
    # tests/ops.rs:984-990
    with pytest.raises(FgfError, match="rows is 30 bytes"):
        ops.mul_add_scatter(Gf8B, buf(30), 8, [1] * 4, buf(8, 64))
    with pytest.raises(FgfError, match="mul_add_scatter: rows is 30 bytes but 4 rows of 8 bytes need 32"):
        ops.mul_add_scatter(Gf8B, buf(30), 8, [1] * 4, buf(8, 64))


def test_matrix_rejects_wrong_coefficient_count():
    # tests/ops.rs:992-998
    with pytest.raises(FgfError, match="coefficients for"):
        ops.mul_add_matrix(Gf8B, buf(32), 8, 4, [([1, 1], buf(8, 64))])


def test_dot_product_matrix_rejects_wrong_coefficient_count():
    # tests/ops.rs:1000-1006
    with pytest.raises(FgfError, match="dot_product_matrix: term supplies 2 coefficients for 4 rows"):
        ops.dot_product_matrix(Gf8B, buf(32), 8, 4, [([1, 1], buf(8, 64))])


def test_matrix_scattered_rejects_overlapping_rows():
    # tests/ops.rs:502-509
    with pytest.raises(FgfError, match="overlap"):
        ops.mul_add_matrix_scattered(Gf8B, buf(64), 16, [0, 8], [([1, 1], buf(16, 128))])


def test_matrix_scattered_rejects_out_of_bounds_row():
    # tests/ops.rs:511-517
    with pytest.raises(FgfError, match="but dst is"):
        ops.mul_add_matrix_scattered(Gf8B, buf(32), 16, [0, 24], [([1, 1], buf(16, 128))])
    with pytest.raises(FgfError, match=r"mul_add_matrix_scattered: row 1 spans 24\.\.40 but dst is 32 bytes"):
        ops.mul_add_matrix_scattered(Gf8B, buf(32), 16, [0, 24], [([1, 1], buf(16, 128))])


def test_matrix_scattered_rejects_wrong_coefficient_count():
    # tests/ops.rs:519-524
    with pytest.raises(FgfError, match="coefficients for"):
        ops.mul_add_matrix_scattered(Gf8B, buf(64), 16, [0, 16, 32], [([1, 1], buf(16, 128))])


def test_matrix_scattered_rejects_misaligned_row():
    with pytest.raises(FgfError, match="offset 3 is not a whole number of"):
        ops.mul_add_matrix_scattered(Gf16, buf(64), 16, [3], [([1], buf(16, 128))])


def test_gather_messages():
    with pytest.raises(FgfError, match="mul_add_gather: 2 coefficients for 1 sources"):
        ops.mul_add_gather(Gf8D, buf(8), [2, 3], [buf(8, 64)])
    with pytest.raises(FgfError, match="mul_add_gather: source is 4 bytes, expected 8"):
        ops.mul_add_gather(Gf8D, buf(8), [2], [buf(4, 64)])


def test_matrix_source_length_message():
    with pytest.raises(FgfError, match="mul_add_matrix: source is 7 bytes, expected 8"):
        ops.mul_add_matrix(Gf8B, buf(32), 8, 4, [([1, 1, 1, 1], buf(7, 64))])


def test_elementwise_messages():
    with pytest.raises(FgfError, match="mul_elementwise: dst is 8 bytes but a is 4 bytes"):
        ops.mul_elementwise(Gf8B, buf(8), buf(4, 64), buf(8, 128))
    with pytest.raises(FgfError, match="mul_elementwise: dst is 8 bytes but b is 6 bytes"):
        ops.mul_elementwise(Gf8B, buf(8), buf(8, 64), buf(6, 128))


def test_plan_matrix_counts():
    # ops.rs:198-212
    with pytest.raises(FgfError, match=r"Plan::matrix: 3 coefficients for 2x2 matrix"):
        ops.Plan.matrix(Gf8B, 2, 2, [1, 2, 3])
