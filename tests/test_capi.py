"""The C-ABI library loads and exports every function include/pga_b200.h
declares (no GPU needed: nothing is called)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "pga_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pga_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header():
    from distributedpanga_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_product_fails_loudly_without_library(monkeypatch):
    from distributedpanga_b200 import pipeline
    monkeypatch.setattr(pipeline, "LIB_PATH", "/nonexistent/libpga_b200.so")
    monkeypatch.setattr(pipeline, "_LIB", None)
    import pytest
    with pytest.raises(RuntimeError):
        pipeline.load_library()
