"""The bit-sliced GF(2) tensor-core kernel (gf2mma.cu), forced on every shape
it covers, against the CPU oracle bit for bit (tolerance 0: the arithmetic is
exact). Shapes: k * E <= 64 input bytes and m * E <= 16 output bytes per
element column, i.e. up to Gf8 RS(64,16), Gf16 RS(32,8), Gf32 RS(16,4);
lengths of one 512-column block, several blocks plus a ragged tail, an
unaligned head, and more blocks than SMs (persistent CTAs reusing the source
ring); overwrite, accumulate and scattered rows; prepared plans and raw
coefficients. After every call the kernel's bounded waits must not have run
out (fgfc_device_check)."""
import numpy as np
import pytest
import torch

from fgf_b200 import _lib, ops, tune
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32
from oracle import orc

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _force_gf2mma(cuda):
    tune.force("gf2mma")
    yield
    tune.force("auto")


def _device_ok():
    st = _lib.lib().fgfc_device_check(1)
    assert st == 0, _lib.lib().fgfc_last_error().decode()


def _coeffs(field, n, rng, nonzero=False):
    lo = 1 if nonzero else 0
    return [int(x) for x in rng.integers(lo, 1 << (8 * field.BYTES), size=n, dtype=np.uint64)]


def _run_case(field, k, m, ncols, head_off=0, seed=1, kind="dot", with_plan=True):
    """ncols element columns per row; every source and row starts head_off
    bytes past a 16-byte boundary (a multiple of the element size)."""
    rng = np.random.default_rng(seed)
    E = field.BYTES
    L = ncols * E
    stride = (L + head_off + 16 + 255) // 256 * 256
    pool = torch.from_numpy(rng.integers(0, 256, size=(k + m + 1) * stride, dtype=np.uint8)).cuda()
    srcs = [pool[t * stride + head_off:t * stride + head_off + L] for t in range(k)]
    vals = _coeffs(field, k * m, rng)
    host_srcs = [s.cpu().numpy().copy() for s in srcs]
    if kind == "scatter":
        gap = (L + 16 + 15) // 16 * 16 + 16
        base = pool[k * stride + head_off:]
        dst = base[:gap * m]
        starts = [j * gap for j in range(m)][::-1]
        want = dst.cpu().numpy().copy()
        orc.mul_add_matrix_scattered(field.ID, want, L, starts, vals, host_srcs)
        if with_plan:
            ops.mul_add_matrix_scattered_with(dst, L, starts, ops.Plan.matrix(field, k, m, vals), srcs)
        else:
            ops.mul_add_matrix_scattered(field, dst, L, starts, [(vals[t * m:(t + 1) * m], srcs[t]) for t in range(k)])
    else:
        # rows j * L apart share the sources' alignment when L is a multiple of 16
        rows = torch.from_numpy(rng.integers(0, 256, size=m * L + 16 + head_off, dtype=np.uint8)).cuda()
        dst = rows[head_off:head_off + m * L]
        want = dst.cpu().numpy().copy()
        if kind == "dot":
            orc.dot_product_matrix(field.ID, want, L, m, vals, host_srcs)
            if with_plan:
                ops.dot_product_matrix_with(dst, L, m, ops.Plan.matrix(field, k, m, vals), srcs)
            else:
                ops.dot_product_matrix(field, dst, L, m, [(vals[t * m:(t + 1) * m], srcs[t]) for t in range(k)])
        else:
            orc.mul_add_matrix(field.ID, want, L, m, vals, host_srcs)
            if with_plan:
                ops.mul_add_matrix_with(dst, L, m, ops.Plan.matrix(field, k, m, vals), srcs)
            else:
                ops.mul_add_matrix(field, dst, L, m, [(vals[t * m:(t + 1) * m], srcs[t]) for t in range(k)])
    torch.cuda.synchronize()
    _device_ok()
    got = dst.cpu().numpy()
    assert np.array_equal(got, want), (
        f"{field.__name__} k={k} m={m} cols={ncols} head={head_off} {kind}: "
        f"{int(np.count_nonzero(got != want))} bytes differ from the oracle")


SHAPES = [
    (Gf8D, 10, 4), (Gf8B, 64, 16), (Gf8D, 1, 1), (Gf8D, 3, 5), (Gf8B, 13, 7), (Gf8D, 64, 1), (Gf8D, 1, 16),
    (Gf16, 32, 8), (Gf16, 5, 3), (Gf16, 1, 1), (Gf16, 31, 1),
    (Gf32, 16, 4), (Gf32, 3, 1), (Gf32, 1, 2), (Gf32, 7, 3),
]


@pytest.mark.parametrize("field,k,m", SHAPES, ids=lambda x: getattr(x, "__name__", str(x)))
def test_one_block_and_ragged_tail(field, k, m):
    assert tune.chosen(field, k, m, 4096) == "gf2mma"
    _run_case(field, k, m, 512, seed=k * 31 + m)             # exactly one block
    _run_case(field, k, m, 3 * 512 + 48, seed=k * 37 + m)     # 3 blocks, then a table-kernel tail
    _run_case(field, k, m, 2 * 512 + 37, seed=k * 41 + m)     # rows of mixed alignment: tables only


@pytest.mark.parametrize("field,k,m", [(Gf8D, 10, 4), (Gf16, 6, 3), (Gf32, 5, 2)],
                         ids=lambda x: getattr(x, "__name__", str(x)))
def test_unaligned_head(field, k, m):
    _run_case(field, k, m, 4 * 512 + 16, head_off=4, seed=5)  # 12 head bytes and the tail on the table path


@pytest.mark.parametrize("field,k,m", [(Gf8D, 4, 2), (Gf16, 4, 4), (Gf32, 2, 2), (Gf8B, 20, 9)],
                         ids=lambda x: getattr(x, "__name__", str(x)))
def test_many_blocks_per_cta(field, k, m):
    # 1000 blocks over at most 148 CTAs: every CTA cycles its 4-stage ring and
    # both TMEM buffers many times
    _run_case(field, k, m, 1000 * 512, seed=9)


@pytest.mark.parametrize("kind", ["add", "scatter"])
@pytest.mark.parametrize("with_plan", [True, False], ids=["plan", "raw"])
def test_accumulate_and_scattered(kind, with_plan):
    _run_case(Gf8D, 10, 4, 8 * 512, seed=11, kind=kind, with_plan=with_plan)
    _run_case(Gf16, 12, 5, 8 * 512 + 5, seed=12, kind=kind, with_plan=with_plan)
    _run_case(Gf32, 9, 3, 8 * 512, seed=13, kind=kind, with_plan=with_plan)


def test_raw_coefficient_form():
    _run_case(Gf8B, 64, 16, 2 * 512, seed=14, with_plan=False)
    _run_case(Gf16, 32, 8, 2 * 512 + 1, seed=15, with_plan=False)


def test_single_row_ops_that_qualify():
    """mul_add_scatter with 16 rows and mul_add_gather with 64 sources run the
    scatter / gather orientations of a plan through the same kernel."""
    rng = np.random.default_rng(16)
    L = 6 * 512
    src = torch.from_numpy(rng.integers(0, 256, size=L, dtype=np.uint8)).cuda()
    rows = torch.from_numpy(rng.integers(0, 256, size=16 * L, dtype=np.uint8)).cuda()
    c = _coeffs(Gf8D, 16, rng)
    want = rows.cpu().numpy().copy()
    orc.mul_add_scatter(Gf8D.ID, want, L, c, src.cpu().numpy().copy())
    ops.mul_add_scatter_with(rows, L, ops.Plan.new(Gf8D, c), src)
    torch.cuda.synchronize()
    _device_ok()
    assert np.array_equal(rows.cpu().numpy(), want)
    srcs = [torch.from_numpy(rng.integers(0, 256, size=L, dtype=np.uint8)).cuda() for _ in range(64)]
    dst = torch.from_numpy(rng.integers(0, 256, size=L, dtype=np.uint8)).cuda()
    c = _coeffs(Gf8D, 64, rng)
    want = dst.cpu().numpy().copy()
    orc.mul_add_gather(Gf8D.ID, want, c, [s.cpu().numpy().copy() for s in srcs])
    ops.mul_add_gather_with(dst, ops.Plan.new(Gf8D, c), srcs)
    torch.cuda.synchronize()
    _device_ok()
    assert np.array_equal(dst.cpu().numpy(), want)


def test_outside_its_range_falls_back():
    """65 sources or 17 Gf8 rows exceed one contraction: the table kernels run."""
    assert not tune.usable("gf2mma", Gf8D, 65, 4)
    assert not tune.usable("gf2mma", Gf8D, 4, 17)
    assert not tune.usable("gf2mma", Gf16, 33, 1)
    assert tune.chosen(Gf8D, 65, 4, 1 << 20) == "nibble"
    _run_case(Gf8D, 65, 2, 2 * 512, seed=17)


def test_tuner_measures_and_records(tmp_path):
    tune.force("auto")
    tune.clear()
    best = tune.tune_shape(Gf16, 32, 8, 1 << 20)
    assert best in ("nibble", "gf2mma")
    assert tune.chosen(Gf16, 32, 8, 1 << 20) == best
    tune.save(str(tmp_path / "t.json"))
    tune.clear()
    tune.load(str(tmp_path / "t.json"))
    assert tune.chosen(Gf16, 32, 8, 1 << 20) == best
    tune.clear()
    _device_ok()
