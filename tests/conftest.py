"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and call the
product through its C ABI; everything else runs on the CPU."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)

GOLDEN_CASES = ["small_s002", "chromset_s0005", "edge_mix", "many_contigs"]
# golden cases whose inputs are regenerated from the seeded generator
REGENERATED = {"small_full": ("small", 1.0), "chromset_full": ("chromset", 1.0), "full_s001": ("full", 0.01),
               "pangenome_s002": ("pangenome", 0.02)}
# large golden cases (digests only, tests/helpers.py check_*_large)
LARGE_CASES = [c for c in ("full_s001", "pangenome_s002", "chromset_full")
               if os.path.exists(os.path.join(GOLDEN, c + ".json"))]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU; calls the product through its C ABI")


def load_case(name: str):
    from distributedpanga_b200 import gdb, synth
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        dig = json.load(f)
    if name in REGENERATED:
        wl, scale = REGENERATED[name]
        cs = gdb.from_contigs(synth.make(wl, scale=scale))
    else:
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        cs = gdb.ContigSet(bps=z["bps"], clen=z["clen"], boff=z["boff"], freq=z["freq"])
    import hashlib
    h = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    assert h(cs.bps) + h(cs.clen) + h(cs.boff) == dig["input_sha"], "golden input drifted: " + name
    return cs, dig


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.build()
    return binding


@pytest.fixture(scope="session")
def dev():
    from distributedpanga_b200 import build, pipeline
    build.build()
    d = pipeline.Device(0)
    yield d
    d.close()
