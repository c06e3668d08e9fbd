"""The C-ABI library loads and exports every entry point include/lbibcell.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "lbibcell.h")).read()
    return sorted(set(re.findall(r"^\s*int\s+(lbib_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "lbib_create_from_files" in syms and "lbib_step" in syms
    assert len(syms) >= 10


def test_library_exports_declared_symbols():
    from lbibcell_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from lbibcell_b200 import build
        build.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    for s in declared_symbols():
        assert hasattr(L, s), s
    assert set(declared_symbols()) >= set(_lib.SYMBOLS)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from lbibcell_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.load()
