"""Kernel-family choice (tune.cpp) on the host: the override, usability per
shape, and the JSON table round trip. No GPU needed."""
import json

import pytest

from fgf_b200 import tune
from fgf_b200._lib import FgfError
from fgf_b200.fields import Gf8B, Gf8D, Gf16, Gf32


@pytest.fixture(autouse=True)
def _reset():
    tune.force("auto")
    tune.clear()
    yield
    tune.force("auto")
    tune.clear()


def test_byte_tables_only_for_gf8_up_to_4_rows_and_14_sources():
    assert tune.usable("byte", Gf8D, 10, 4)
    assert tune.usable("byte", Gf8B, 14, 1)
    assert not tune.usable("byte", Gf8D, 15, 4)
    assert not tune.usable("byte", Gf8D, 10, 5)
    assert not tune.usable("byte", Gf16, 10, 2)
    for f in (Gf8B, Gf8D, Gf16, Gf32):
        assert tune.usable("nibble", f, 64, 16)


def test_builtin_rule_and_override():
    assert tune.chosen(Gf8D, 10, 4, 4 << 20) == "byte"      # long rows: byte tables
    assert tune.chosen(Gf8D, 10, 4, 64 << 10) == "nibble"   # short rows: tables fill faster
    tune.force("nibble")
    assert tune.chosen(Gf8D, 10, 4, 4 << 20) == "nibble"
    tune.force("byte")
    assert tune.chosen(Gf16, 8, 2, 4 << 20) != "byte"       # never forced onto a shape it cannot run
    tune.force("auto")
    assert tune.chosen(Gf8D, 10, 4, 4 << 20) == "byte"


def test_variants_list_the_choice_first():
    v = tune.variants_for(Gf8D, 10, 4, 4 << 20)
    assert v[0] == "byte" and "nibble" in v


def test_table_round_trip(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text('{"version": 1, "entries": [\n'
                    '  {"field": 1, "k": 10, "m": 4, "len_log2": 16, "kernel": "byte", "us": 3.250}\n]}\n')
    tune.load(str(path))
    assert tune.chosen(Gf8D, 10, 4, 1 << 16) == "byte"       # measured winner beats the built-in rule
    assert tune.chosen(Gf8D, 10, 4, 1 << 15) == "nibble"     # other buckets keep the rule
    out = tmp_path / "out.json"
    tune.save(str(out))
    data = json.loads(out.read_text())
    assert data["entries"] == [{"field": 1, "k": 10, "m": 4, "len_log2": 16, "kernel": "byte", "us": 3.25}]


def test_tiles_set_get_and_round_trip(tmp_path):
    """Work-list tile shapes: built-in 8 columns per thread, settable per
    (element width, groups) class, persisted beside the family table."""
    assert tune.tile(2, 4) == 8
    tune.set_tile(2, 4, 2)
    tune.set_tile(1, 1, 16)
    assert (tune.tile(2, 4), tune.tile(1, 1), tune.tile(4, 1)) == (2, 16, 8)
    p = tmp_path / "tune.json"
    tune.save(str(p))
    doc = json.loads(p.read_text())
    assert sorted((t["elem_bytes"], t["groups"], t["cols"]) for t in doc["tiles"]) == [(1, 1, 16), (2, 4, 2)]
    tune.clear()
    assert tune.tile(2, 4) == 8
    tune.load(str(p))
    assert (tune.tile(2, 4), tune.tile(1, 1)) == (2, 16)
    tune.set_tile(2, 4, 0)
    assert tune.tile(2, 4) == 8


@pytest.mark.parametrize("args", [(3, 1, 8), (2, 5, 8), (2, 0, 8), (2, 2, 3), (1, 1, 32)])
def test_tiles_refuse_unknown_classes_and_shapes(args):
    with pytest.raises(FgfError):
        tune.set_tile(*args)
