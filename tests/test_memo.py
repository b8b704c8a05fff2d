"""The served form's table of a target's recorded Local_Alignment calls
(distributedpanga_b200/csrc/memo.h) on the host: every distinct logged call
whose trace was kept is found with its first value, a call whose trace was
not kept and a call never logged are not, and the table stays at most half
full (tests/native/memo_check.cpp)."""
import os
import subprocess

from conftest import ROOT

NATIVE = os.path.join(ROOT, "tests", "native")


def test_memo_table():
    src = os.path.join(NATIVE, "memo_check.cpp")
    hdr = os.path.join(ROOT, "distributedpanga_b200", "csrc", "memo.h")
    exe = os.path.join(NATIVE, "memo_check")
    if not os.path.exists(exe) or max(os.path.getmtime(src), os.path.getmtime(hdr)) > os.path.getmtime(exe):
        subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Werror", "-o", exe, src], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("ok n=") == 5, out.stdout
