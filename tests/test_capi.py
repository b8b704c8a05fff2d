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


def test_dropin_driver_defines_reference_signatures():
    """The reference's driver linked with the drop-in stages (built by
    `make -C oracle dropin` where the reference tree is present) defines
    every function include/pga_dropin.h declares itself -- none comes from a
    reference source -- and loads libpga_b200.so."""
    import subprocess
    import pytest
    exe = os.path.join(ROOT, "oracle", "_ref", "pga-mpi-merge-b200")
    if not os.path.exists(exe):
        pytest.skip("the drop-in driver is not built here (no reference tree)")
    txt = open(os.path.join(ROOT, "include", "pga_dropin.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", txt)))
    assert len(names) >= 20
    syms = subprocess.run(["nm", exe], check=True, capture_output=True, text=True).stdout
    defined = {l.split()[-1] for l in syms.split("\n") if len(l.split()) == 3 and l.split()[1] in "TtDdBb"}
    missing = [n for n in names if n not in defined]
    assert not missing, missing
    # the drop-in file is where they are defined
    src = open(os.path.join(ROOT, "distributedpanga_b200", "dropin", "pga_dropin.c")).read()
    assert all(re.search(r"\b%s\s*\(" % n, src) for n in names)
    ldd = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    assert "libpga_b200.so" in ldd


def test_wrappers_marshal_their_arguments():
    """Wrappers whose entry points return before touching a device when the
    context is null: their arguments marshal through the declared ctypes
    signatures (no ArgumentError) and the library answers PGA_ERR_ARG."""
    import numpy as np
    import pytest
    from distributedpanga_b200 import pipeline
    d = object.__new__(pipeline.Device)
    d.L = pipeline.load_library()
    d.h = None
    d.nseeds = [0, 0]
    calls = [d.reuse_stats, d.alloc_times, d.stage_times, d.align_stats, d.align_times,
             lambda: d.seeds_load(0, np.zeros(7, np.uint8))]
    for call in calls:
        with pytest.raises(pipeline.PgaError):
            call()
