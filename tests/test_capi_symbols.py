"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from turbogap_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(?:int|const char\s*\*|void)\s+\**\s*(tgx?_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_headers_declare_entry_points():
    names = declared_symbols()
    assert "tg_get_gap_soap" in names and "tg_soap_begin" in names
    assert "tg_build_neighbors_list" in names and "tg_engine_md" in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.fail("libtgb200.so is not built (python -m turbogap_b200.build)")
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(L, n)]
    assert not missing, missing


def test_python_signatures_cover_headers():
    sig = {n for n, _, _ in _lib.SIGNATURES}
    assert declared_symbols() <= sig
