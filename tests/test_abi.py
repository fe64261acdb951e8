"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(mstmg_[a-z0-9_]+)\s*\(", txt):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ["mstmg_ctx_create", "mstmg_ctx_destroy", "mstmg_interaction", "mstmg_bicg", "mstmg_fixed_orientation",
              "mstmg_planewave"]:
        assert n in names


def test_library_exports_all_declared_symbols():
    from mstm_b200 import _lib
    from mstm_b200 import build as B
    if not os.path.exists(_lib.LIB_PATH):
        B.build()
    L = _lib.lib()
    for n in declared_symbols():
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, n


def test_missing_library_fails_loudly(monkeypatch):
    from mstm_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libmstm_b200.so")
    with pytest.raises(RuntimeError):
        _lib.lib()
