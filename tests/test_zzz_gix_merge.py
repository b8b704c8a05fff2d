"""GIXmake's index on disk into the GPU merge: read by pga_read_gix, merged
by pga_self_adaptamer_merge and diagonal sorted on the device, the seeds
and panels are the reference's (golden digests), although GIXmake leaves
runs of equal k-mers in its own order.

This file is collected last so that a run stopping at the first failure has
run every other test before it."""
import os
import tempfile

import pytest

from conftest import GOLDEN_CASES, load_case
from helpers import check_diag, check_seeds
from test_gix import HAVE_GIXMAKE, gixmake

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not HAVE_GIXMAKE, reason="oracle/_ref not built")
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_gixmake_index_through_the_gpu_merge(dev, case):
    from distributedpanga_b200 import pipeline
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    with tempfile.TemporaryDirectory() as work:
        g = pipeline.read_gix(gixmake(cs, work))
    assert (g["post_bytes"], g["cont_bytes"]) == (posb, ctgb)
    dev.gdb_load(cs)
    ns, css, nb, cb = dev.self_adaptamer_merge(g["entries"], g["cum"], posb, ctgb, dig["freq_cutoff"],
                                               cs.ncontig)
    check_seeds(ns, css, nb, cb, dig)
    for u, seeds in (("N", ns), ("C", css)):
        arr, off = dev.reimport_sort(seeds, posb, ctgb, 1 if u == "C" else 0, cs.ncontig, cs.maxctg, dig["dbyte"])
        check_diag(arr, off, u, dig)
