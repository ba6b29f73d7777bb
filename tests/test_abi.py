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
