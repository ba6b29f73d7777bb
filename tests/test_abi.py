"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import re
from pathlib import Path

from fgf_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared(header: str) -> set[str]:
    text = (ROOT / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(fgfc_[a-z0-9_]+)\s*\(", text))


def test_header_declares_the_ops_surface():
    names = declared("fgf_cuda.h")
    for op in ("mul_add", "mul_add_with", "mul_add_scatter", "mul_add_scatter_with", "mul_add_gather",
               "mul_add_gather_with", "dot_product", "dot_product_with", "mul_add_matrix",
               "mul_add_matrix_with", "dot_product_matrix", "dot_product_matrix_with",
               "mul_add_matrix_scattered", "plan_create", "plan_destroy"):
        assert f"fgfc_{op}" in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    for header in sorted(p.name for p in (ROOT / "include").glob("*.h")):
        for name in sorted(declared(header)):
            assert hasattr(lib, name), f"{name} declared in include/{header} but not exported"


def test_binding_covers_the_header():
    assert declared("fgf_cuda.h") <= set(_lib.declared_symbols())


def test_rust_crate_binds_every_entry_point():
    """The fgf-cuda crate (source only here: no cargo in this image) declares
    every C-ABI entry point in sys.rs and mirrors every public fgf::ops
    function (src/ops.rs:323-1017) in ops.rs."""
    crate = ROOT / "fgf_b200" / "rust" / "fgf-cuda" / "src"
    sys_rs = (crate / "sys.rs").read_text()
    bound = set(re.findall(r"pub fn (fgfc_[a-z0-9_]+)\s*\(", sys_rs))
    missing = declared("fgf_cuda.h") - bound
    assert not missing, f"sys.rs lacks {sorted(missing)}"
    ops_rs = (crate / "ops.rs").read_text()
    wrapped = set(re.findall(r"pub fn ([a-z_]+)<F: CudaField>", ops_rs))
    for op in ("add_assign", "sub_assign", "mul_add", "mul_add_with", "mul_into", "mul_into_with", "mul_assign",
               "mul_assign_with", "mul_elementwise", "mul_add_scatter", "mul_add_scatter_with", "mul_add_gather",
               "mul_add_gather_with", "dot_product", "dot_product_with", "mul_add_matrix", "mul_add_matrix_with",
               "dot_product_matrix", "dot_product_matrix_with", "mul_add_matrix_scattered"):
        assert op in wrapped, f"ops.rs lacks {op}"


def test_field_codes_agree_across_header_python_and_rust():
    """fgfc_field codes: the header enum, the Python field markers and the
    crate's constants and CudaField impls name the same fields."""
    from fgf_b200.fields import FIELDS

    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "fgf_cuda.h").read_text(), flags=re.S)
    enum = {name: int(v) for name, v in re.findall(r"\b(FGFC_(?:GF|FP)[0-9A-Z]+)\s*=\s*(\d+)", text)}
    sys_rs = (ROOT / "fgf_b200" / "rust" / "fgf-cuda" / "src" / "sys.rs").read_text()
    rust = {name: int(v) for name, v in re.findall(r"pub const (FGFC_(?:GF|FP)[0-9A-Z]+): fgfc_field = (\d+);", sys_rs)}
    assert enum == rust
    assert sorted(enum.values()) == sorted(FIELDS)
    ops_rs = (ROOT / "fgf_b200" / "rust" / "fgf-cuda" / "src" / "ops.rs").read_text()
    impls = set(re.findall(r"const ID: sys::fgfc_field = sys::(FGFC_[0-9A-Z]+);", ops_rs))
    assert impls == set(enum)
