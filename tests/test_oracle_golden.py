"""The oracle restatement against golden digests of the reference pipeline
(tests/golden, made by running the reference compiled from source)."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_case
from helpers import check_diag, check_index, check_seeds, sha


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_oracle_matches_reference(oracle, case):
    cs, dig = load_case(case)
    assert sha(cs.bps) + sha(cs.clen) + sha(cs.boff) == dig["input_sha"]
    posb, ctgb = dig["posb"], dig["ctgb"]
    rec = oracle.extract(cs, posb, ctgb)
    srt = oracle.sort_records(rec)
    check_index(srt, dig)
    ent, cum, big = oracle.build_adapter(srt, posb, ctgb)
    ns, css, nb, cb = oracle.merge(ent, cum, posb, ctgb, dig["freq_cutoff"], cs.ncontig)
    check_seeds(ns, css, nb, cb, dig)
    for u, seeds in (("N", ns), ("C", css)):
        arr, off = oracle.reimport_sort(seeds, posb, ctgb, 1 if u == "C" else 0, cs.ncontig,
                                        cs.maxctg, dig["dbyte"])
        check_diag(arr, off, u, dig)
