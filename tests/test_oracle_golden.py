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


def test_oracle_matches_reference_large(oracle):
    """The 20 Mbp sample of the 2 x 1 Gbp generator (40 % interspersed
    repeats, tandem arrays, 7,241 contigs with 2-byte contig fields): every
    stage of the restatement against the reference's digests."""
    from helpers import check_diag_large, check_index_large, check_seeds_large
    cs, dig = load_case("full_s001")
    posb, ctgb = dig["posb"], dig["ctgb"]
    srt = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    check_index_large(srt, dig)
    ent, cum, _ = oracle.build_adapter(srt, posb, ctgb)
    del srt
    ns, css, nb, cb = oracle.merge(ent, cum, posb, ctgb, dig["freq_cutoff"], cs.ncontig)
    del ent
    check_seeds_large(ns, css, nb, cb, dig)
    for u, seeds in (("N", ns), ("C", css)):
        arr, off = oracle.reimport_sort(seeds, posb, ctgb, 1 if u == "C" else 0, cs.ncontig,
                                        cs.maxctg, dig["dbyte"])
        check_diag_large(arr, off, u, dig)
