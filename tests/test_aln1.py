"""The .1aln writer (pga_write_1aln): files it writes read back, through the
reference's own ONE reader (oracle/_ref/alndump, open_Aln_Read), as the
reference's alignment record stream and GDB skeleton."""
import gzip
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, ROOT, load_case

ALNDUMP = os.path.join(ROOT, "oracle", "_ref", "alndump")
needs_ref = pytest.mark.skipif(not os.path.exists(ALNDUMP), reason="oracle/_ref not built")


def parse_lines(lines):
    """alndump text -> (recs9, toff, trace) as pga_align_copy gives them."""
    recs, toff, tr = [], [0], []
    for l in lines:
        head, T, X = l.split(";")
        a = [int(x) for x in head.split()]
        T = [int(x) for x in T.split()]
        X = [int(x) for x in X.split()]
        assert len(T) == len(X)
        recs.append(a + [2 * len(T)])
        for d, b in zip(X, T):
            tr += [d, b]
        toff.append(len(tr))
    # alndump order: aread abpos aepos bread bbpos bepos comp diffs
    return (np.array(recs, dtype=np.int32).reshape(-1, 9), np.array(toff, dtype=np.int64),
            np.array(tr, dtype=np.uint8))


def dump(path, skel=False):
    out = subprocess.run([ALNDUMP] + (["-s"] if skel else []) + [path], check=True, capture_output=True,
                         text=True).stdout
    return [" ".join(l.split()) for l in out.split("\n") if l.strip() and not l.startswith("#")]


@needs_ref
@pytest.mark.parametrize("case", GOLDEN_CASES + ["small_full"])
def test_written_file_reads_back_as_reference_stream(case):
    from distributedpanga_b200 import pipeline
    cs, dig = load_case(case)
    ref = [" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n")
           if l.strip()]
    recs, toff, tr = parse_lines(ref)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "out.1aln")
        pipeline.write_1aln(p, recs, toff, tr, cs.clen, db_name="g.1gdb", cwd=d)
        got = dump(p)
    assert len(got) == dig["aln"]["count"]
    assert got == ref


@needs_ref
def test_skeleton_and_records_equal_reference_file():
    """The reference's own .1aln for a small contig set and the file written
    here from its records and the FASTA's contigs read back identically,
    skeleton included."""
    from distributedpanga_b200 import pipeline, synth
    from oracle import binding as B
    contigs = synth.make("small", scale=0.02)
    with tempfile.TemporaryDirectory() as d:
        fa = os.path.join(d, "g.fa")
        synth.write_fasta(fa, contigs)
        B.ref_make_gdb(fa, os.path.join(d, "g"))
        out = B.ref_run(os.path.join(d, "g"), d)
        ref_full = dump(out["aln"], skel=True)
        ref_recs = [l for l in ref_full if ";" in l]
        recs, toff, tr = parse_lines(ref_recs)
        p = os.path.join(d, "mine.1aln")
        pipeline.write_1aln(p, recs, toff, tr, [len(c) for c in contigs], db_name="g.1gdb", cwd=d)
        mine_full = dump(p, skel=True)
    assert len(ref_recs) > 0
    assert any(l.startswith("S ") for l in ref_full)
    assert mine_full == ref_full


def test_writer_rejects_bad_arguments():
    from distributedpanga_b200 import pipeline
    L = pipeline.load_library()
    assert L.pga_write_1aln(b"/tmp/x.1aln", None, b"v", b"c", b"db", None, 100, 0, None, None, None, None, None,
                            0, None, None, None) == 2
