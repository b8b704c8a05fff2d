"""The bench's roofline arithmetic on CPU: the index build's algorithmic
bytes (ceil(G/4) + 5*N*R + N*E + 2^27, E = R - 3), the aligner's cells per
second, the served form's summary object and the per-workload cutoffs."""
import sys

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    import bench as b
    return b


def test_index_bytes_formula(bench):
    from distributedpanga_b200 import gdb
    rng = np.random.default_rng(3)
    cs = gdb.from_contigs([rng.integers(0, 4, n).astype(np.uint8) for n in (70_000, 1_234, 300_001)])
    posb, ctgb, rsize = gdb.record_sizing(cs)
    assert rsize == 12 + posb + ctgb
    n = 123_457
    want = (cs.seqtot + 3) // 4 + 5 * n * rsize + n * (rsize - 3) + (1 << 27)
    assert bench.index_bytes(cs, n, True) == want
    assert bench.index_bytes(cs, n, False) == want - n * (rsize - 3)


def test_align_roofline_cells_per_second(bench):
    r = bench.align_roofline({"cells": 466_375_070, "waves": 28_094_913, "calls": 12_195, "tasks": 384_211}, 320.0)
    assert r["bound"] == "issue" and r["unit"] == "cells/s"
    assert r["achieved"] == pytest.approx(466_375_070 / 0.320)
    assert bench.align_roofline({"cells": 1, "waves": 1, "calls": 1, "tasks": 1}, 0.0)["achieved"] is None


def test_serve_compact_and_cutoffs(bench):
    keep = ("p50_latency_s", "p99_latency_s", "gdb_mbp_per_s", "query_mbp_per_s", "wall_s")
    summ = {k: float(i) for i, k in enumerate(keep)}
    m = {"value": 1.5, "config": {"workload": "w", "slots": 3}, "served": dict(summ, extra=1),
         "plain": dict(summ, extra=2), "served_over_plain": 1.1, "bit_exact_requests": "12/12",
         "call_record": {"requests_using_it": 11}, "clocks": {"sm_mhz": 1965.0}}
    c = bench.serve_compact(m)
    assert c["served"] == summ and c["plain"] == summ and c["bit_exact_requests"] == "12/12"
    assert c["call_record"] == {"requests_using_it": 11}
    assert c["slots"] == 3 and c["value"] == 1.5
    old = bench.WL["name"]
    try:
        bench.WL["name"] = "chromset"
        assert bench.freq_cutoff() == 10
        bench.WL["name"] = "pangenome"
        assert bench.freq_cutoff() == 10    # the reference driver's cutoff (src/pga-mpi-merge.c:62)
    finally:
        bench.WL["name"] = old
