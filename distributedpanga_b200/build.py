"""Builds the sm_100a shared library libpga_b200.so in-tree with nvcc.

``python -m distributedpanga_b200.build`` (or ``build()``) compiles every
``csrc/*.cu`` for ``arch=compute_100a,code=sm_100a`` with ``-lineinfo`` into
``distributedpanga_b200/libpga_b200.so``; the library exports the C ABI
of ``include/pga_b200.h``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpga_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def sources() -> list:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [
        os.path.join(ROOT, "include", "pga_b200.h")]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    cmd = [NVCC, *FLAGS, "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp", *sources()]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(HERE, "csrc", "ptxas.log")
    with open(log, "w") as f:
        f.write(res.stdout)
        f.write(res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stderr[-8000:])
        raise RuntimeError("nvcc failed (see %s)" % log)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        sys.stderr.write(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
