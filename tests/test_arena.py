"""The context's device arena (distributedpanga_b200/csrc/arena.h) on the
host against a fake device: placement, alignment, coalescing, best fit,
returning empty slabs when the device is full, and repeated pipeline passes
with the buffer sizes of a 2 x 1 Gbp genome pair that make driver calls only
in the first pass (tests/native/arena_check.cpp)."""
import os
import subprocess

from conftest import ROOT

NATIVE = os.path.join(ROOT, "tests", "native")


def test_arena_checks():
    src = os.path.join(NATIVE, "arena_check.cpp")
    hdr = os.path.join(ROOT, "distributedpanga_b200", "csrc", "arena.h")
    exe = os.path.join(NATIVE, "arena_check")
    if not os.path.exists(exe) or max(os.path.getmtime(src), os.path.getmtime(hdr)) > os.path.getmtime(exe):
        subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Werror", "-o", exe, src], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.split("\n")
    assert any(x.startswith("ok pipeline_passes") and "later=0" in x for x in lines), out.stdout
