"""The rule pga_serve_load builds a request's GDB by: GDB(target text +
query text) is the target's GDB followed by the query's, the query's contig
byte offsets moved by the target's image, its scaffold numbers by the
target's scaffolds, its scaffolds' contig ranges by the target's contigs and
their header offsets by the target's header bytes, the base counts summed.
Checked here against Create_GDB's reader (the oracle) on every ordered pair of
the FASTA edge cases; the GPU test (tests/test_serve.py) checks the device
code against the device ingest of the concatenated text."""
import itertools

import numpy as np
import pytest

from fasta_cases import CASES, NTHR


def splice(t: dict, q: dict) -> dict:
    qc = q["contigs"].copy()
    qc[:, 1] += len(t["bps"])
    qc[:, 3] += t["nscaff"]
    qs = q["scaffolds"].copy()
    qs[:, 0] += t["ncontig"]
    qs[:, 1] += t["ncontig"]
    qs[:, 3] += len(t["headers"])
    return {"contigs": np.concatenate([t["contigs"], qc]), "scaffolds": np.concatenate([t["scaffolds"], qs]),
            "headers": t["headers"] + q["headers"], "bps": np.concatenate([t["bps"], q["bps"]]),
            "count": t["count"] + q["count"], "maxctg": max(t["maxctg"], q["maxctg"]),
            "seqtot": t["seqtot"] + q["seqtot"]}


def _check(oracle, ta: bytes, qa: bytes, nthr: int):
    t, q, both = oracle.fasta_gdb(ta, nthr), oracle.fasta_gdb(qa, nthr), oracle.fasta_gdb(ta + qa, nthr)
    s = splice(t, q)
    for k in ("contigs", "scaffolds", "bps", "count"):
        assert np.array_equal(s[k], both[k]), k
    assert s["headers"] == both["headers"]
    assert s["maxctg"] == both["maxctg"] and s["seqtot"] == both["seqtot"]


def test_splice_every_pair_of_cases(oracle):
    texts = {k: f() for k, f in CASES.items()}
    for a, b in itertools.product(sorted(texts), repeat=2):
        _check(oracle, texts[a], texts[b], 0)


@pytest.mark.parametrize("nthr", [n for n in NTHR if n])
def test_splice_with_gap_thresholds(oracle, nthr):
    texts = {k: f() for k, f in CASES.items()}
    for a, b in [("runs", "gap_lengths"), ("gap_lengths", "runs"), ("scaffold_boundaries", "runs_across_lines"),
                 ("crlf", "blank_lines"), ("many_scaffolds", "headers")]:
        _check(oracle, texts[a], texts[b], nthr)
