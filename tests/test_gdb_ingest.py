"""GDB ingest: Create_GDB's FASTA reader (lib/GDB.c:771-1057).

The oracle (oracle/pga_oracle.c orc_fasta_gdb) is pinned to the reference's
own reader through tests/golden/fasta_edge.npz (made by fa2gdb + gdbdump, see
tests/golden/make_fasta_golden.py) and, where oracle/_ref is built, live on
fresh random texts.  The GPU ingest is checked against both, bit for bit:
contig and scaffold tables, header block, base frequencies, .bps image.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import tempfile

import numpy as np
import pytest

import fasta_cases as FC
from conftest import GOLDEN, ROOT

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
HAVE_REF = all(os.path.exists(os.path.join(REF_DIR, x)) for x in ("fa2gdb", "gdbdump"))
PARAMS = [(c, t) for c in FC.CASES for t in FC.NTHR]


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(GOLDEN, "fasta_edge.npz"))


def expect(golden, case, nthr):
    k = "%s.%d." % (case, nthr)
    return {x: golden[k + x] for x in ("text_sha", "contigs", "scaffolds", "names", "freq", "bps_sha")}


def check_tables(got_contigs, got_scaffolds, got_headers, got_freq, got_bps, exp):
    assert np.array_equal(got_contigs, exp["contigs"])
    assert np.array_equal(got_scaffolds, exp["scaffolds"])
    # the header block holds the names in scaffold order, each ended by NUL
    assert bytes(got_headers) == exp["names"].tobytes()
    assert np.array_equal(np.asarray(got_freq, np.float32), exp["freq"])
    assert sha(got_bps) == str(exp["bps_sha"])


def oracle_freq(o):
    return (o["count"] / o["seqtot"]).astype(np.float32)


# ---- the oracle against the reference -------------------------------------------

@pytest.mark.parametrize("case,nthr", PARAMS)
def test_oracle_matches_reference_golden(golden, oracle, case, nthr):
    text = FC.CASES[case]()
    exp = expect(golden, case, nthr)
    assert sha(text) == str(exp["text_sha"]), "FASTA generator drifted"
    o = oracle.fasta_gdb(text, nthr)
    check_tables(o["contigs"], o["scaffolds"], o["headers"], oracle_freq(o), o["bps"], exp)


@pytest.mark.parametrize("name", sorted(FC.ERRORS))
def test_oracle_rejects_what_reference_rejects(golden, oracle, name):
    assert bool(golden[name + ".rejected"])
    with pytest.raises(ValueError):
        oracle.fasta_gdb(FC.ERRORS[name], 0)


def reference_gdb(text: bytes, nthr: int, work: str):
    from oracle import binding as B
    fa = os.path.join(work, "in.fa")
    with open(fa, "wb") as f:
        f.write(text)
    stem = os.path.join(work, "g")
    B.ref_make_gdb(fa, stem, nthr)
    return B.ref_gdb_tables(stem)


def as_expected(r):
    names = np.frombuffer(b"".join(n.encode("latin-1") + b"\0" for n in r["names"]), np.uint8)
    return {"contigs": r["contigs"], "scaffolds": r["scaffolds"], "names": names, "freq": r["freq"],
            "bps_sha": sha(r["bps"].tobytes())}


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("seed,nthr", [(1, 0), (2, 0), (3, 10), (4, 300)])
def test_oracle_matches_reference_live(oracle, seed, nthr):
    text = FC.random_fasta(seed, 400_000)
    with tempfile.TemporaryDirectory() as work:
        r = reference_gdb(text, nthr, work)
    o = oracle.fasta_gdb(text, nthr)
    check_tables(o["contigs"], o["scaffolds"], o["headers"], oracle_freq(o), o["bps"], as_expected(r))


@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
@pytest.mark.parametrize("case", ["runs", "headers", "many_scaffolds", "crlf"])
def test_1gdb_writer_read_by_reference(oracle, case):
    """pga_write_1gdb (host only) on the oracle's tables; the reference's
    Read_GDB reads back the same GDB and .bps."""
    from distributedpanga_b200 import pipeline as P
    L = P.load_library()
    text = FC.CASES[case]()
    o = oracle.fasta_gdb(text, 0)
    freq = oracle_freq(o)
    with tempfile.TemporaryDirectory() as work:
        tpath = os.path.join(work, "w.1gdb")
        hdr = np.frombuffer(o["headers"], np.uint8).copy()
        ctg = np.ascontiguousarray(o["contigs"])
        scf = np.ascontiguousarray(o["scaffolds"])
        bps = o["bps"] if o["bps"].size else np.zeros(1, np.uint8)
        rc = L.pga_write_1gdb(tpath.encode(), b"test", b"0.1", b"test", b"/src/in.fa", freq.ctypes.data,
                              o["nscaff"], scf.ctypes.data, hdr.ctypes.data, hdr.size, o["ncontig"],
                              ctg.ctypes.data, bps.ctypes.data, o["bps"].size)
        assert rc == 0
        from oracle import binding as B
        r = B.ref_gdb_tables(os.path.join(work, "w"))
    check_tables(o["contigs"], o["scaffolds"], o["headers"], freq, o["bps"], as_expected(r))


# ---- the GPU ingest ------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("case,nthr", PARAMS)
def test_ingest_matches_reference(dev, oracle, golden, case, nthr):
    text = FC.CASES[case]()
    exp = expect(golden, case, nthr)
    t = dev.gdb_ingest_fasta(text, nthr)
    check_tables(t.contigs, t.scaffolds, t.headers, t.freq, t.bps, exp)
    o = oracle.fasta_gdb(text, nthr)
    assert np.array_equal(t.bps, o["bps"])
    assert np.array_equal(t.count, o["count"])
    assert t.maxctg == o["maxctg"]


@pytest.mark.gpu
def test_ingest_errors(dev):
    from distributedpanga_b200.pipeline import PgaError
    bad = dict(FC.ERRORS)
    bad["nul"] = b">a\nAC\x00GT\n"
    bad["non_ascii"] = b">a\nAC\xc3\xa9GT\n"
    bad["non_ascii_header"] = b">\xff\nACGT\n"
    for name, text in bad.items():
        with pytest.raises(PgaError):
            dev.gdb_ingest_fasta(text, 0)
    # the context stays usable
    t = dev.gdb_ingest_fasta(b">ok\nACGTN\nA\n", 0)
    assert t.contigs.tolist() == [[4, 0, 0, 0], [1, 1, 5, 0]]


@pytest.mark.gpu
@pytest.mark.parametrize("seed,nthr,mb", [(21, 0, 48), (22, 20, 24), (23, 0, 3)])
def test_ingest_large_matches_oracle(dev, oracle, seed, nthr, mb):
    """Tens of MB with scaffolds of lognormal size, N runs and lower case:
    every table and the .bps image equal the oracle's."""
    text = FC.random_fasta(seed, mb << 20)
    t = dev.gdb_ingest_fasta(text, nthr)
    o = oracle.fasta_gdb(text, nthr)
    assert np.array_equal(t.contigs, o["contigs"])
    assert np.array_equal(t.scaffolds, o["scaffolds"])
    assert t.headers == o["headers"]
    assert np.array_equal(t.bps, o["bps"])
    assert np.array_equal(t.count, o["count"])


@pytest.mark.gpu
@pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")
def test_ingest_written_gdb_read_by_reference(dev):
    text = FC.random_fasta(5, 2 << 20)
    t = dev.gdb_ingest_fasta(text, 0)
    with tempfile.TemporaryDirectory() as work:
        dev.gdb_write(os.path.join(work, "d.1gdb"), "/src/in.fa")
        from oracle import binding as B
        r = B.ref_gdb_tables(os.path.join(work, "d"))
        with tempfile.TemporaryDirectory() as w2:
            ref = reference_gdb(text, 0, w2)
    check_tables(t.contigs, t.scaffolds, t.headers, t.freq, t.bps, as_expected(r))
    check_tables(t.contigs, t.scaffolds, t.headers, t.freq, t.bps, as_expected(ref))


def golden_fasta(cs) -> bytes:
    """The FASTA the golden cases were made from (synth.write_fasta: one
    scaffold ctg<i> per contig, 80 bases a line)."""
    letters = np.frombuffer(b"ACGT", np.uint8)
    out = []
    for i in range(cs.ncontig):
        s = letters[cs.contig(i)].tobytes()
        out.append(b">ctg%d\n" % i + b"".join(s[j:j + 80] + b"\n" for j in range(0, len(s), 80)))
    return b"".join(out)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["small_s002", "edge_mix"])
def test_fasta_to_alignments_on_gpu(dev, case):
    """FASTA text -> GDB -> index -> seeds -> alignments, all on the device:
    the GDB is the reference's and the alignments are its .1aln records."""
    import gzip
    from conftest import load_case
    from distributedpanga_b200.pipeline import alignment_lines
    cs, dig = load_case(case)
    t = dev.gdb_ingest_fasta(golden_fasta(cs), 0)
    assert np.array_equal(t.bps, cs.bps)
    assert np.array_equal(t.contigs[:, 0], cs.clen) and np.array_equal(t.contigs[:, 1], cs.boff)
    assert np.array_equal(t.freq, cs.freq)
    dev.index_build(want_entries=False)
    dev.merge(dig["freq_cutoff"])
    dev.set_ranges(0)
    n = dev.align()
    mine = [" ".join(l.split()) for l in alignment_lines(*dev.alignments())]
    ref = [" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n")
           if l.strip()]
    assert n == dig["aln"]["count"]
    assert mine == ref


def gapped_fasta(seed: int) -> bytes:
    """The small workload at scale 0.02 (2 x 40 kbp) joined into scaffolds of
    one to three contigs with N gaps between them (scaffold 1 and some others
    open with N's, scaffold 2 and some others end with them), 70 bases a
    line."""
    from distributedpanga_b200 import synth
    rng = np.random.default_rng(seed)
    letters = np.frombuffer(b"ACGT", np.uint8)
    contigs = synth.make("small", scale=0.02)
    out, i, k = [], 0, 0
    while i < len(contigs):
        m = int(rng.integers(1, 4))
        parts = []
        if k == 1 or rng.random() < 0.2:     # an empty first contig
            parts.append(b"N" * int(rng.integers(1, 30)))
        for j, c in enumerate(contigs[i:i + m]):
            if j:
                parts.append(b"N" * int(rng.integers(1, 200)))
            parts.append(letters[c].tobytes())
        if k == 2 or rng.random() < 0.2:     # a dropped trailing run
            parts.append(b"n" * int(rng.integers(1, 30)))
        s = b"".join(parts)
        out.append(b">scaffold_%d some text\n" % k + b"".join(s[x:x + 70] + b"\n" for x in range(0, len(s), 70)))
        i += m
        k += 1
    return b"".join(out)


@pytest.mark.gpu
@pytest.mark.skipif(not all(os.path.exists(os.path.join(REF_DIR, x))
                            for x in ("fa2gdb", "pga-mpi-merge", "GIXmake_dump", "alndump")),
                    reason="oracle/_ref not built")
def test_fasta_with_gaps_to_1aln_matches_reference(dev):
    """FASTA with gapped scaffolds -> GDB -> alignments -> .1aln, every step on
    the GPU, equal to the reference's own pipeline on the same FASTA: the
    record stream and the GDB skeleton (scaffold names, gaps, contigs) read
    back by the reference's ONE reader."""
    from oracle import binding as B
    text = gapped_fasta(7)
    alndump = os.path.join(REF_DIR, "alndump")

    def dump(path):
        out = subprocess.run([alndump, "-s", path], check=True, capture_output=True, text=True).stdout
        return [" ".join(l.split()) for l in out.split("\n") if l.strip() and not l.startswith("#")]

    with tempfile.TemporaryDirectory() as d:
        fa = os.path.join(d, "g.fa")
        with open(fa, "wb") as f:
            f.write(text)
        B.ref_make_gdb(fa, os.path.join(d, "g"))
        ref = dump(B.ref_run(os.path.join(d, "g"), d)["aln"])
        t = dev.gdb_ingest_fasta(text, 0)
        assert t.contigs.shape[0] > t.scaffolds.shape[0]      # gaps split scaffolds
        dev.index_build(want_entries=False)
        dev.merge(10)
        dev.set_ranges(0)
        dev.align()
        p = os.path.join(d, "mine.1aln")
        dev.write_1aln(p, skeleton=t.skeleton(), db_name="g.1gdb", cwd=d)
        mine = dump(p)
    assert sum(";" in l for l in ref) > 0
    assert any(l.startswith("G ") for l in ref)
    assert mine == ref
