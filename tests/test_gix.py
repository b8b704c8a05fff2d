"""The GIX writer (pga_write_gix / pga_index_write_gix): GIXmake's .gix and
.ktab parts (notes/GIXmake_annotated.c:1529-1615) from the k-mer index.

Pinned to GIXmake itself, compiled here from notes/GIXmake_dump.c
(oracle/_ref/GIXmake_dump), on the golden cases: the .gix header, the 2^24
prefix table and the contig order are equal byte for byte; the k-mer table
entries are equal row for row once the runs of equal k-mers are put in one
order (GIXmake leaves them in an unspecified one, so its own tools compare
them that way), leaving out the first entry of each part (GIXmake picks its
part boundaries by sampling).
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN_CASES, ROOT, load_case

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
HAVE_GIXMAKE = all(os.path.exists(os.path.join(REF_DIR, x)) for x in ("fa2gdb", "GIXmake_dump"))


def read_gix(stem: str) -> dict:
    d, r = os.path.split(stem)
    with open(stem + ".gix", "rb") as f:
        b = f.read()
    K, NP, one, three = np.frombuffer(b[:16], np.int32)
    cum = np.frombuffer(b[16:16 + 8 * (1 << 24)], np.int64)
    o = 16 + 8 * (1 << 24)
    pb, cb, np2 = (int(x) for x in np.frombuffer(b[o:o + 12], np.int32))
    o += 12
    maxp = int(np.frombuffer(b[o:o + 8], np.int64)[0])
    o += 8
    freq, nctg = (int(x) for x in np.frombuffer(b[o:o + 8], np.int32))
    o += 8
    perm = np.frombuffer(b[o:o + 4 * nctg], np.int32)
    o += 4 * nctg
    end = int(np.frombuffer(b[o:o + 8], np.int64)[0])
    assert o + 8 == len(b)
    parts = []
    for p in range(1, int(NP) + 1):
        with open(os.path.join(d, ".%s.ktab.%d" % (r, p)), "rb") as f:
            x = f.read()
        k = int(np.frombuffer(x[:4], np.int32)[0])
        n = int(np.frombuffer(x[4:12], np.int64)[0])
        eb = 9 + pb + cb
        assert k == 40 and len(x) == 12 + n * eb
        parts.append(np.frombuffer(x[12:], np.uint8).reshape(-1, eb))
    return {"head": (int(K), int(NP), int(one), int(three), pb, cb, np2, maxp, freq, nctg, end),
            "cum": cum, "perm": perm, "parts": parts}


def canonical(E: np.ndarray) -> np.ndarray:
    """Runs of equal k-mers (bytes 0..7) ordered by payload; the run's LCP on
    its first row, 40 on the others."""
    key = [E[:, j] for j in range(E.shape[1] - 1, 8, -1)] + [E[:, j] for j in range(7, -1, -1)]
    E = E[np.lexsort(key)].copy()
    if len(E) == 0:
        return E
    start = np.ones(len(E), bool)
    start[1:] = np.any(E[1:, :8] != E[:-1, :8], axis=1)
    rid = np.cumsum(start) - 1
    low = np.full(rid[-1] + 1, 255, np.int64)
    np.minimum.at(low, rid, E[:, 8].astype(np.int64))
    E[:, 8] = np.where(start, low[rid], 40).astype(np.uint8)
    return E


def part_starts(parts) -> list:
    return list(np.cumsum([0] + [len(p) for p in parts])[:-1])


def write_from_oracle(oracle, cs, stem, nparts=8):
    from distributedpanga_b200 import gdb, pipeline
    posb, ctgb, _ = gdb.record_sizing(cs)
    rec = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    ent, cum, big = oracle.build_adapter(rec, posb, ctgb)
    order = np.argsort(-cs.clen, kind="stable").astype(np.int32)
    e = np.ascontiguousarray(ent).reshape(-1)
    if e.size == 0:
        e = np.zeros(1, np.uint8)
    rc = pipeline.load_library().pga_write_gix(stem.encode(), nparts, posb, ctgb, cs.ncontig, order.ctypes.data,
                                               cum.ctypes.data, big, ent.shape[0], e.ctypes.data)
    assert rc == 0


def gixmake(cs, work: str) -> str:
    from oracle import binding as B
    letters = np.frombuffer(b"ACGT", np.uint8)
    fa = os.path.join(work, "g.fa")
    with open(fa, "wb") as f:
        for i in range(cs.ncontig):
            s = letters[cs.contig(i)].tobytes()
            f.write(b">ctg%d\n" % i + b"".join(s[j:j + 80] + b"\n" for j in range(0, len(s), 80)))
    B.ref_make_gdb(fa, os.path.join(work, "g"))
    # One thread: with -T8, on a loaded host, GIXmake now and then writes one
    # entry's LCP against the wrong predecessor (seen once in ~30 runs under
    # load: 6 where the first base differs); its parts are the same with -T1.
    subprocess.run([os.path.join(REF_DIR, "GIXmake_dump"), "-T1", os.path.join(work, "g.1gdb")], check=True,
                   capture_output=True, cwd=work)
    return os.path.join(work, "g")


def check_against_gixmake(mine: dict, ref: dict):
    assert mine["head"] == ref["head"]
    assert np.array_equal(mine["cum"], ref["cum"])
    assert np.array_equal(mine["perm"], ref["perm"])
    M, R = np.concatenate(mine["parts"]), np.concatenate(ref["parts"])
    assert M.shape == R.shape
    for i in part_starts(mine["parts"]) + part_starts(ref["parts"]):
        if i < len(M):
            M[i, 8] = R[i, 8] = 255
    assert np.array_equal(canonical(M), canonical(R))


@pytest.mark.skipif(not HAVE_GIXMAKE, reason="oracle/_ref not built")
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_writer_matches_gixmake(oracle, case):
    cs, _ = load_case(case)
    with tempfile.TemporaryDirectory() as work:
        ref = read_gix(gixmake(cs, work))
        os.makedirs(os.path.join(work, "m"))
        write_from_oracle(oracle, cs, os.path.join(work, "m", "g"), nparts=ref["head"][1])
        check_against_gixmake(read_gix(os.path.join(work, "m", "g")), ref)


def test_part_start_lcp_rule(oracle):
    """The first entry of a part carries 0 when the part's first panel holds
    k-mers, else the bases its panel shares with that panel (what GIXmake's
    part-by-part sort leaves, lib/MSDsort.c:485-500); elsewhere the LCP bytes
    are the index's."""
    from distributedpanga_b200 import gdb
    cs, _ = load_case("edge_mix")
    posb, ctgb, _ = gdb.record_sizing(cs)
    rec = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    ent, cum, _ = oracle.build_adapter(rec, posb, ctgb)
    with tempfile.TemporaryDirectory() as work:
        write_from_oracle(oracle, cs, os.path.join(work, "g"), nparts=16)
        g = read_gix(os.path.join(work, "g"))
    M = np.concatenate(g["parts"])
    starts = set(int(i) for i in part_starts(g["parts"]))
    rest = np.array([i for i in range(len(M)) if i not in starts])
    assert np.array_equal(M[rest, 8], ent[rest, 8])
    pstart = np.concatenate([[0], cum[(np.arange(1, 1025) << 14) - 1]])
    for i in starts:
        if i >= len(M):
            continue
        # the part's first panel: the lowest panel whose entries start at i
        q0 = int(np.searchsorted(pstart, i, side="left"))
        q = int(np.searchsorted(pstart, i, side="right")) - 1    # the panel entry i is in
        if q == q0:
            want = 0
        elif (q & 0x300) != (q0 & 0x300):
            want = 0
        else:
            v, z = (q ^ q0) & 0xff, 0
            while z < 4 and not v & (0xc0 >> (2 * z)):
                z += 1
            want = 1 + z
        assert M[i, 8] == want


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["small_s002", "edge_mix", "many_contigs"])
def test_index_gix_equals_oracle_gix(dev, oracle, case):
    """The GIX written from the GPU index is byte for byte the one written
    from the oracle's index (same writer, same parts), and matches GIXmake."""
    cs, _ = load_case(case)
    dev.gdb_load(cs)
    dev.index_build(want_entries=True)
    with tempfile.TemporaryDirectory() as work:
        os.makedirs(os.path.join(work, "gpu"))
        os.makedirs(os.path.join(work, "orc"))
        dev.index_write_gix(os.path.join(work, "gpu", "g"), 8)
        write_from_oracle(oracle, cs, os.path.join(work, "orc", "g"), nparts=8)
        names = sorted(os.listdir(os.path.join(work, "orc")))
        assert names == sorted(os.listdir(os.path.join(work, "gpu")))
        for n in names:
            with open(os.path.join(work, "gpu", n), "rb") as a, open(os.path.join(work, "orc", n), "rb") as b:
                assert a.read() == b.read(), n
        if HAVE_GIXMAKE:
            ref = read_gix(gixmake(cs, work))
            if ref["head"][1] == 8:
                check_against_gixmake(read_gix(os.path.join(work, "gpu", "g")), ref)


# ---- the reader (pga_read_gix): a GIX on disk as the k-mer table view

def _oracle_table(oracle, cs):
    from distributedpanga_b200 import gdb
    posb, ctgb, _ = gdb.record_sizing(cs)
    rec = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    return oracle.build_adapter(rec, posb, ctgb), posb, ctgb


@pytest.mark.parametrize("case,nparts", [("small_s002", 1), ("edge_mix", 16), ("many_contigs", 8),
                                         ("chromset_s0005", 1024)])
def test_reader_inverts_writer(oracle, case, nparts):
    """Written by pga_write_gix and read back by pga_read_gix, the k-mer
    table is the index's, entry for entry: contigs numbered as in the GDB
    again, and every part's first LCP byte the LCP to the entry before it."""
    from distributedpanga_b200 import pipeline
    cs, _ = load_case(case)
    (ent, cum, big), posb, ctgb = _oracle_table(oracle, cs)
    with tempfile.TemporaryDirectory() as work:
        write_from_oracle(oracle, cs, os.path.join(work, "g"), nparts=nparts)
        g = pipeline.read_gix(os.path.join(work, "g"))
    assert (g["kmer"], g["parts"], g["post_bytes"], g["cont_bytes"], g["freq"]) == (40, nparts, posb, ctgb, 0)
    assert np.array_equal(g["order"], np.argsort(-cs.clen, kind="stable"))
    assert np.array_equal(g["cum"], cum) and g["largest"] == big
    assert np.array_equal(g["entries"], ent)


@pytest.mark.skipif(not HAVE_GIXMAKE, reason="oracle/_ref not built")
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_reader_on_gixmake_output(oracle, case):
    """GIXmake's own index, read by pga_read_gix, is the oracle's k-mer table
    once runs of equal k-mers are put in one order (GIXmake leaves them in an
    unspecified one), part starts included."""
    from distributedpanga_b200 import pipeline
    cs, _ = load_case(case)
    (ent, cum, big), _, _ = _oracle_table(oracle, cs)
    with tempfile.TemporaryDirectory() as work:
        g = pipeline.read_gix(gixmake(cs, work))
    assert np.array_equal(g["cum"], cum)
    assert np.array_equal(g["order"], np.argsort(-cs.clen, kind="stable"))
    assert np.array_equal(canonical(g["entries"].copy()), canonical(ent.copy()))


def test_reader_rejects_bad_files():
    from distributedpanga_b200 import pipeline
    with tempfile.TemporaryDirectory() as work:
        with pytest.raises(pipeline.PgaError):
            pipeline.read_gix(os.path.join(work, "missing"))
        with open(os.path.join(work, "short.gix"), "wb") as f:
            f.write(np.array([40, 1, 1, 3], np.int32).tobytes())
        with pytest.raises(pipeline.PgaError):
            pipeline.read_gix(os.path.join(work, "short"))


@pytest.mark.skipif(not HAVE_GIXMAKE, reason="oracle/_ref not built")
@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_gixmake_index_feeds_the_merge(oracle, case):
    """The k-mer table read from GIXmake's files is a merge input like the
    built index's: merged (the oracle's adaptamer merge stands in for
    pga_self_adaptamer_merge, which takes the same table; its GPU run is in
    test_zzz_gix_merge.py) and diagonal sorted, its seeds and N and C
    panels are the reference's (golden digests)."""
    from helpers import check_diag, check_seeds
    from distributedpanga_b200 import pipeline
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    with tempfile.TemporaryDirectory() as work:
        g = pipeline.read_gix(gixmake(cs, work))
    ns, css, nb, cb = oracle.merge(g["entries"], g["cum"], posb, ctgb, dig["freq_cutoff"], cs.ncontig)
    check_seeds(ns, css, nb, cb, dig)
    for u, seeds in (("N", ns), ("C", css)):
        arr, off = oracle.reimport_sort(seeds, posb, ctgb, 1 if u == "C" else 0, cs.ncontig, cs.maxctg,
                                        dig["dbyte"])
        check_diag(arr, off, u, dig)


def test_reader_rejects_corrupt_indexes(oracle):
    """A GIX damaged in each field the reader trusts -- the .gix cut short,
    a contig order that is not a permutation, a part that claims more
    entries than the prefix table holds, a contig place past the last
    contig, a part missing -- is refused with an error, never read past
    its buffers."""
    import shutil
    from distributedpanga_b200 import pipeline
    cs, _ = load_case("edge_mix")
    with tempfile.TemporaryDirectory() as work:
        good = os.path.join(work, "good")
        os.makedirs(good)
        write_from_oracle(oracle, cs, os.path.join(good, "g"), nparts=4)
        g = pipeline.read_gix(os.path.join(good, "g"))
        eb = 9 + g["post_bytes"] + g["cont_bytes"]
        order_at = 16 + 8 * (1 << 24) + 12 + 8 + 8

        def damaged(name, edit):
            d = os.path.join(work, name)
            shutil.copytree(good, d)
            edit(d)
            with pytest.raises(pipeline.PgaError):
                pipeline.read_gix(os.path.join(d, "g"))

        def patch(path, at, data):
            with open(path, "r+b") as f:
                f.seek(at)
                f.write(data)

        damaged("short", lambda d: os.truncate(os.path.join(d, "g.gix"), order_at))
        damaged("perm", lambda d: patch(os.path.join(d, "g.gix"), order_at + 4,
                                        np.int32(g["order"][0]).tobytes()))
        damaged("count", lambda d: patch(os.path.join(d, ".g.ktab.1"), 4, np.int64(1 << 40).tobytes()))
        place = np.zeros(g["cont_bytes"], np.uint8)
        place[:] = 0xff
        place[-1] = 0x7f
        damaged("place", lambda d: patch(os.path.join(d, ".g.ktab.2"), 12 + 9 + g["post_bytes"], place.tobytes()))
        damaged("missing", lambda d: os.remove(os.path.join(d, ".g.ktab.3")))
