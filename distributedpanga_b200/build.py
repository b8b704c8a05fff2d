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
         "-Xcompiler", "-fPIC", "-Xptxas", "-v"]


def sources() -> list:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers() -> list:
    return (glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(HERE, "csrc", "*.h"))
            + [os.path.join(ROOT, "include", "pga_b200.h")])


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in sources() + headers())


def _compile(src: str, obj: str) -> subprocess.CompletedProcess:
    cmd = [NVCC, *FLAGS, "-c", "-I", os.path.join(ROOT, "include"), "-o", obj, src]
    return subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every translation unit in parallel (one nvcc each, objects in
    csrc/_build/), then links the shared library.  A unit is recompiled when
    it or any header is newer than its object."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    odir = os.path.join(HERE, "csrc", "_build")
    os.makedirs(odir, exist_ok=True)
    newest_header = max(os.path.getmtime(h) for h in headers())
    jobs = []
    for src in sources():
        obj = os.path.join(odir, os.path.basename(src)[:-3] + ".o")
        stale = force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src),
                                                                                   newest_header)
        jobs.append((src, obj, stale))
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4)) as ex:
        futs = {src: ex.submit(_compile, src, obj) for src, obj, stale in jobs if stale}
        results = {src: f.result() for src, f in futs.items()}
    log = os.path.join(HERE, "csrc", "ptxas.log")
    with open(log, "w") as f:
        for src, res in sorted(results.items()):
            f.write("==== %s\n" % os.path.basename(src))
            f.write(res.stdout)
            f.write(res.stderr)
    bad = [src for src, res in results.items() if res.returncode != 0]
    if bad:
        for src in bad:
            sys.stderr.write(results[src].stderr[-8000:])
        raise RuntimeError("nvcc failed on %s (see %s)" % (", ".join(os.path.basename(b) for b in bad), log))
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-fPIC",
            "-o", LIB + ".tmp", *[obj for _, obj, _ in jobs]]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stderr[-8000:])
        raise RuntimeError("nvcc link failed")
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        for res in results.values():
            sys.stderr.write(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
