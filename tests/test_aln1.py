"""The .1aln writers (pga_write_1aln, ONE's ASCII encoding, and
pga_write_1aln_binary, its binary one): files they write read back, through
the reference's own ONE reader (oracle/_ref/alndump, open_Aln_Read), as the
reference's alignment record stream and GDB skeleton; a binary file's footer
(counts, list sizes, per-object statistics, the objects' byte index) reads
back as the reference's own binary file's does (oracle/_ref/onestat)."""
import gzip
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, ROOT, load_case

ALNDUMP = os.path.join(ROOT, "oracle", "_ref", "alndump")
ONESTAT = os.path.join(ROOT, "oracle", "_ref", "onestat")
needs_ref = pytest.mark.skipif(not os.path.exists(ALNDUMP) or not os.path.exists(ONESTAT),
                               reason="oracle/_ref not built")


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


def stat(path):
    return subprocess.run([ONESTAT, path], check=True, capture_output=True, text=True).stdout.split("\n")


@needs_ref
@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("case", GOLDEN_CASES + ["small_full"])
def test_written_file_reads_back_as_reference_stream(case, binary):
    from distributedpanga_b200 import pipeline
    cs, dig = load_case(case)
    ref = [" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n")
           if l.strip()]
    recs, toff, tr = parse_lines(ref)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "out.1aln")
        pipeline.write_1aln(p, recs, toff, tr, cs.clen, db_name="g.1gdb", cwd=d, binary=binary)
        got = dump(p)
        st = stat(p)
    assert len(got) == dig["aln"]["count"]
    assert got == ref
    assert st[0] == "binary %d" % binary
    if binary:  # every alignment reached through the index, last first
        assert [l.split()[3:] for l in st if l.startswith("@ A ")] == [l.split()[:6] for l in reversed(ref)]


@needs_ref
@pytest.mark.parametrize("kind,scale", [("small", 0.02), ("pangenome", 0.01)])
def test_skeleton_and_records_equal_reference_file(kind, scale):
    """The reference's own .1aln for a contig set and the files written here
    from its records and the FASTA's contigs read back identically, skeleton
    included; the binary one's footer reads back as the reference's does.
    The pan-genome's trace lists pass the 100,000 bytes after which the
    reference's ONElib codes them, and the binary file here codes them too
    (its codec built from all of them): it is no larger than the
    reference's."""
    from distributedpanga_b200 import pipeline, synth
    from oracle import binding as B
    contigs = synth.make(kind, scale=scale)
    with tempfile.TemporaryDirectory() as d:
        fa = os.path.join(d, "g.fa")
        synth.write_fasta(fa, contigs)
        B.ref_make_gdb(fa, os.path.join(d, "g"))
        out = B.ref_run(os.path.join(d, "g"), d)
        ref_full = dump(out["aln"], skel=True)
        ref_stat = stat(out["aln"])
        ref_recs = [l for l in ref_full if ";" in l]
        recs, toff, tr = parse_lines(ref_recs)
        mine = {}
        for binary in (False, True):
            p = os.path.join(d, "mine%d.1aln" % binary)
            pipeline.write_1aln(p, recs, toff, tr, [len(c) for c in contigs], db_name="g.1gdb", cwd=d,
                                binary=binary)
            mine[binary] = (dump(p, skel=True), stat(p))
        sizes = (os.path.getsize(out["aln"]), os.path.getsize(os.path.join(d, "mine1.1aln")))
    assert len(ref_recs) > 0
    assert any(l.startswith("S ") for l in ref_full)
    assert ref_stat[0] == "binary 1"
    assert mine[False][0] == ref_full
    assert mine[True][0] == ref_full
    assert mine[True][1] == ref_stat
    if kind == "pangenome":
        assert sizes[1] <= sizes[0], sizes


@needs_ref
@pytest.mark.parametrize("regime", ["few", "many", "constant"])
def test_binary_encoding_edges(regime):
    """Values at every width of ONE's variable-length integers, trace lists of
    0, 1 and many values whose differences need one or two bytes, scaffolds
    with leading, inner and trailing gaps and one of gap alone, and files
    with no skeleton or no
    alignments: the binary file reads back as the ASCII one does, and its
    index reaches every object.  "few" stays below the size at which trace
    lists are coded; "many" codes them (differences of one and two bytes,
    lists left uncoded where coding does not pay); "constant" codes lists
    whose bytes are all one value (a one-symbol code)."""
    from distributedpanga_b200 import pipeline
    rng = np.random.default_rng(7)
    widths = [0, 1, 63, 64, 8191, 8192, 65535, 65536, 2 ** 24 - 1, 2 ** 24, 2 ** 31 - 1]
    recs, toff, tr = [], [0], []
    for i, v in enumerate(widths * (3 if regime == "few" else 40)):
        n = [0, 1, 2, 37, 200][i % 5]
        if regime == "constant":
            t = np.full(2 * n, 100)
        else:
            t = rng.integers(0, 256, 2 * n) if i % 2 else rng.integers(0, 40, 2 * n)
        recs.append([i % 4, v, v, (i + 1) % 4, widths[(i + 3) % len(widths)], v, i % 2, v, 2 * n])
        tr += t.tolist()
        toff.append(len(tr))
    recs = np.array(recs, dtype=np.int64).clip(0, 2 ** 31 - 1).astype(np.int32)
    toff = np.array(toff, dtype=np.int64)
    tr = np.array(tr, dtype=np.uint8)
    clen = np.array([2 ** 33, 70, 9000, 5], dtype=np.int64)
    sk = pipeline.Skeleton(["chr with space", "b" * 300, "c", "all gap"], [2 ** 33 + 100, 10000, 5, 77],
                           [0, 1, 3, 4, 4], [100, 0, 500, 0])
    with tempfile.TemporaryDirectory() as d:
        for skel, n in ((sk, len(recs)), (sk, 0), (None, len(recs))):
            got = {}
            for binary in (False, True):
                p = os.path.join(d, "e%d.1aln" % binary)
                pipeline.write_1aln(p, recs[:n], toff[:n + 1], tr, clen, skeleton=skel, db_name="g.1gdb",
                                    binary=binary)
                got[binary] = (dump(p, skel=True), stat(p))
                if binary:  # the footer (at the offset in the last 8 bytes) has the trace codecs or not
                    b = open(p, "rb").read()
                    foot = b[int.from_bytes(b[-8:], "little"):]
                    assert (b"\xe8T" in foot) == (regime != "few" and n > 0)
            assert got[True][0] == got[False][0]
            st = got[True][1]
            assert [int(l.split()[2]) for l in st if l.startswith("@ A ")] == list(range(n, 0, -1))
            assert all("unreachable" not in l for l in st)
            if n:
                assert ("# A %d 0 0" % n) in st


ALNWRITE = os.path.join(ROOT, "oracle", "_ref", "alnwrite")


@needs_ref
@pytest.mark.skipif(not os.path.exists(ALNWRITE), reason="oracle/_ref/alnwrite not built")
@pytest.mark.parametrize("source", ["small_full", "synthetic"])
def test_c_caller_with_reference_types(source):
    """oracle/_ref/alnwrite, a C program holding the alignments in the
    reference's Overlap records and GDB skeleton, writes them through the
    reference's own writer (as la_merge does) and through
    pga_write_1aln_binary: the reference's reader gets the same records,
    skeleton, counts, per-object statistics and index from both files.  The
    synthetic set's lists pass the size at which both writers code them."""
    from distributedpanga_b200 import pipeline
    if source == "small_full":
        cs, _ = load_case(source)
        ref = [" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, source + ".aln.txt.gz"), "rt").read()
               .split("\n") if l.strip()]
        recs, toff, tr = parse_lines(ref)
        clen = cs.clen
        sk = None
    else:
        rng = np.random.default_rng(3)
        recs, toff, tr = [], [0], []
        for i in range(3000):
            n = [0, 1, 2, 37, 200][i % 5]
            t = rng.integers(0, 256, 2 * n) if i % 2 else rng.integers(0, 40, 2 * n)
            recs.append([i % 4, i, i + 5, (i + 1) % 4, 7 * i, 9 * i, i % 2, i % 50, 2 * n])
            tr += t.tolist()
            toff.append(len(tr))
        recs, toff, tr = np.array(recs, np.int32), np.array(toff), np.array(tr, np.uint8)
        clen = [2 ** 33, 70, 9000, 5]
        sk = pipeline.Skeleton(["chr with space", "b" * 300, "c"], [2 ** 33 + 100, 10000, 5], [0, 1, 3, 4],
                               [100, 0, 500, 0])
    with tempfile.TemporaryDirectory() as d:
        src, a, b = (os.path.join(d, f) for f in ("in.1aln", "ref.1aln", "pga.1aln"))
        pipeline.write_1aln(src, recs, toff, tr, clen, skeleton=sk, db_name="g.1gdb", cwd=d)
        subprocess.run([ALNWRITE, src, a, b], check=True, capture_output=True)
        assert dump(a, skel=True) == dump(b, skel=True) == dump(src, skel=True)
        assert stat(a) == stat(b)
        if source == "synthetic":
            assert os.path.getsize(b) <= os.path.getsize(a)


def test_writer_rejects_bad_arguments():
    from distributedpanga_b200 import pipeline
    L = pipeline.load_library()
    for fn in (L.pga_write_1aln, L.pga_write_1aln_binary):
        assert fn(b"/tmp/x.1aln", None, b"v", b"c", b"db", None, 100, 0, None, None, None, None, None,
                  0, None, None, None) == 2
        assert fn(b"/tmp/x.1aln", b"p", b"v", b"c", b"db", None, 0, 0, None, None, None, None, None,
                  0, None, None, None) == 2
