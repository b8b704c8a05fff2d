"""GPU parity on the large golden cases: the benchmarked 2 x 100 Mbp workload
(chromset_full), a 20 Mbp sample of the 2 x 1 Gbp generator (full_s001:
40 % interspersed repeats, tandem arrays, 7,241 contigs) and the pan-genome
generator at 2 % (17 genomes at the reference driver's FREQ = 10).  Every
stage of the resident pipeline -- index, N and C seeds, sorted diagonal
panels, and the .1aln record stream -- against digests of the reference's
own pipeline run on the same seeded inputs (tests/golden/make_golden.py)."""
import pytest

from conftest import LARGE_CASES, load_case
from helpers import check_diag_large, check_index_large, check_lines, check_seeds_large

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", LARGE_CASES)
def test_large_case_matches_reference(dev, case):
    from distributedpanga_b200.pipeline import alignment_lines
    cs, dig = load_case(case)
    dev.gdb_load(cs)
    n = dev.index_build(want_entries=False)
    assert n == dig["index"]["count"]
    rec = dev.index_records()
    check_index_large(rec, dig)
    del rec
    dev.merge(dig["freq_cutoff"])
    ns, nb = dev.seeds(0)
    css, cb = dev.seeds(1)
    check_seeds_large(ns, css, nb, cb, dig)
    del ns, css
    for comp, u in ((0, "N"), (1, "C")):
        sw, cnt = dev.diag_sort(comp)
        assert sw == dig["swide"]
        arr, off = dev.diag_records(comp, sw, cnt)
        check_diag_large(arr, off, u, dig)
        del arr
    dev.align()
    lines = [" ".join(x.split()) for x in alignment_lines(*dev.alignments())]
    check_lines(lines, dig["aln"])
