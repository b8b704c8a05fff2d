"""GPU parity: every stage of the CUDA path through the C ABI, against the
oracle (bit-exact, same order) and the golden digests of the reference."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_case
from helpers import check_diag, check_index, check_seeds

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_dropin_stages(dev, oracle, case):
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    dev.gdb_load(cs)
    assert dev.record_sizing() == (posb, ctgb, dig["rsize"])

    ext = dev.extract_to_records()                      # extract_to_records
    want = oracle.extract(cs, posb, ctgb)
    assert np.array_equal(ext, want)                    # same records, same emission order

    srt = dev.sort_records(ext, posb, ctgb)            # run_stage2: sort + LCP
    check_index(srt, dig)
    assert np.array_equal(srt, oracle.sort_records(want))

    ent, cum, big = dev.build_kmer_adapter(srt, posb, ctgb)
    oent, ocum, obig = oracle.build_adapter(srt, posb, ctgb)
    assert np.array_equal(ent, oent) and np.array_equal(cum, ocum) and big == obig

    ns, css, nb, cb = dev.self_adaptamer_merge(ent, cum, posb, ctgb, dig["freq_cutoff"], cs.ncontig)
    ons, ocs, onb, ocb = oracle.merge(oent, ocum, posb, ctgb, dig["freq_cutoff"], cs.ncontig)
    assert np.array_equal(ns, ons) and np.array_equal(css, ocs)
    assert np.array_equal(nb, onb) and np.array_equal(cb, ocb)
    check_seeds(ns, css, nb, cb, dig)

    for u, seeds in (("N", ns), ("C", css)):
        arr, off = dev.reimport_sort(seeds, posb, ctgb, 1 if u == "C" else 0, cs.ncontig, cs.maxctg,
                                     dig["dbyte"])
        check_diag(arr, off, u, dig)


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_resident_pipeline(dev, oracle, case):
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    dev.gdb_load(cs)
    n = dev.index_build(want_entries=True)
    assert n == dig["index"]["count"]
    srt = dev.index_records()
    check_index(srt, dig)
    osrt = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    assert np.array_equal(srt, osrt)
    ent, cum, big = dev.index_entries()
    oent, ocum, obig = oracle.build_adapter(osrt, posb, ctgb)
    assert np.array_equal(ent, oent) and np.array_equal(cum, ocum) and big == obig
    dev.merge(dig["freq_cutoff"])
    ns, nb = dev.seeds(0)
    css, cb = dev.seeds(1)
    check_seeds(ns, css, nb, cb, dig)
    ons, ocs, _, _ = oracle.merge(oent, ocum, posb, ctgb, dig["freq_cutoff"], cs.ncontig)
    assert np.array_equal(ns, ons) and np.array_equal(css, ocs)
    for comp, u in ((0, "N"), (1, "C")):
        sw, cnt = dev.diag_sort(comp)
        assert sw == dig["swide"]
        arr, off = dev.diag_records(comp, sw, cnt)
        check_diag(arr, off, u, dig)


def test_small_workload_full_size(dev, oracle):
    """The 2 + 2 Mbp workload at full size: every stage bit-exact vs the oracle."""
    from distributedpanga_b200 import gdb, synth
    cs = gdb.from_contigs(synth.make("small"))
    posb, ctgb, rsize = gdb.record_sizing(cs)
    dbyte, swide = gdb.diag_sizing(cs, ctgb)
    dev.gdb_load(cs)
    dev.index_build(want_entries=True)
    srt = dev.index_records()
    osrt = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    assert np.array_equal(srt, osrt)
    dev.merge(10)
    ns, nb = dev.seeds(0)
    css, cb = dev.seeds(1)
    oent, ocum, _ = oracle.build_adapter(osrt, posb, ctgb)
    ons, ocs, onb, ocb = oracle.merge(oent, ocum, posb, ctgb, 10, cs.ncontig)
    assert np.array_equal(ns, ons) and np.array_equal(css, ocs)
    assert np.array_equal(nb, onb) and np.array_equal(cb, ocb)
    for comp, seeds in ((0, ons), (1, ocs)):
        sw, cnt = dev.diag_sort(comp)
        arr, off = dev.diag_records(comp, sw, cnt)
        oarr, ooff = oracle.reimport_sort(seeds, posb, ctgb, comp, cs.ncontig, cs.maxctg, dbyte)
        assert np.array_equal(arr, oarr) and np.array_equal(off, ooff)


def test_degenerate_inputs(dev, oracle):
    from distributedpanga_b200 import gdb
    rng = np.random.default_rng(3)
    # only contigs too short for a 12-mer: no records at all
    cs = gdb.from_contigs([rng.integers(0, 4, n).astype(np.uint8) for n in (1, 5, 11)])
    dev.gdb_load(cs)
    assert dev.index_build() == 0
    assert dev.extract_to_records().shape[0] == 0
    assert dev.merge(10) == (0, 0)
    # a single 12-mer
    cs = gdb.from_contigs([rng.integers(0, 4, 12).astype(np.uint8)])
    posb, ctgb, _ = gdb.record_sizing(cs)
    dev.gdb_load(cs)
    assert np.array_equal(dev.extract_to_records(), oracle.extract(cs, posb, ctgb))


@pytest.mark.parametrize("bits", [0, 19, 20, 22])
def test_index_skewed_digits(dev, oracle, bits):
    """Digits (the first 9 to 11 bases) of every size class of the two-level
    sort: a poly-A run puts ~30,000 records into one digit and one prefix
    bucket (the global path and the bitonic network), tandem copies of a
    9-base unit put thousands into a few digits (the 8192-record shared-memory
    class), random sequence fills the rest.  Equal to the oracle's sorted
    index at the automatic width and at forced wider ones."""
    from distributedpanga_b200 import gdb
    rng = np.random.default_rng(29)
    unit = np.array([0, 1, 2, 3, 3, 2, 1, 0, 3], np.uint8)
    contigs = [np.zeros(30000, np.uint8), np.tile(unit, 5000),
               np.concatenate([np.tile(unit[:5], 3000), rng.integers(0, 4, 500).astype(np.uint8)])]
    contigs += [rng.integers(0, 4, n).astype(np.uint8) for n in (50000, 20000, 777)]
    cs = gdb.from_contigs(contigs)
    posb, ctgb, _ = gdb.record_sizing(cs)
    dev.gdb_load(cs)
    dev.set_digit_bits(bits)
    try:
        n = dev.index_build(want_entries=True)
    finally:
        dev.set_digit_bits(0)
    want = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    assert n == want.shape[0]
    assert np.array_equal(dev.index_records(), want)
    ent, cum, big = dev.index_entries()
    oent, ocum, obig = oracle.build_adapter(want, posb, ctgb)
    assert np.array_equal(ent, oent) and np.array_equal(cum, ocum) and big == obig


def test_sort_matches_property_at_scale(dev):
    """Size-independent properties of the index at 2 x 20 Mbp: sorted order,
    LCPs equal to the recomputed bases-in-common, prefix table consistent."""
    from distributedpanga_b200 import gdb, synth
    cs = gdb.from_contigs(synth.make("chromset", scale=0.2))
    dev.gdb_load(cs)
    n = dev.index_build(want_entries=True)
    rec = dev.index_records()
    assert rec.shape[0] == n
    k = rec[:, 1:11]
    # lexicographic non-decreasing k-mers: (first 8 bytes, last 2 bytes) as big-endian integers
    hi = np.ascontiguousarray(k[:, :8]).view(">u8").reshape(-1)
    lo = (k[:, 8].astype(np.uint32) << 8) | k[:, 9]
    assert np.all((hi[1:] > hi[:-1]) | ((hi[1:] == hi[:-1]) & (lo[1:] >= lo[:-1])))
    # LCP = leading equal bases of neighbours
    x = np.bitwise_xor(k[1:], k[:-1])
    first = np.argmax(x != 0, axis=1)
    allsame = ~np.any(x != 0, axis=1)
    byte = x[np.arange(len(x)), first]
    lead = np.where(byte >= 64, 0, np.where(byte >= 16, 1, np.where(byte >= 4, 2, 3)))
    want = np.where(allsame, 40, 4 * first + lead)
    assert rec[0, 0] == 0 and np.array_equal(rec[1:, 0], want)
    ent, cum, big = dev.index_entries()
    assert cum[-1] == n and big == int(np.max(np.diff(np.concatenate([[0], cum]))))


def _aln_norm(lines):
    return [" ".join(l.split()) for l in lines if l.strip()]


@pytest.mark.parametrize("case", GOLDEN_CASES + ["small_full"])
def test_alignments_match_reference(dev, case):
    """The whole path on the GPU; the .1aln record stream equals the reference's."""
    import gzip
    import os
    from conftest import GOLDEN
    from distributedpanga_b200.pipeline import alignment_lines
    cs, dig = load_case(case)
    dev.gdb_load(cs)
    dev.index_build(want_entries=False)
    dev.merge(dig["freq_cutoff"])
    dev.set_ranges(0)
    n = dev.align()
    recs, toff, tr = dev.alignments()
    mine = _aln_norm(alignment_lines(recs, toff, tr))
    ref = _aln_norm(gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n"))
    assert n == dig["aln"]["count"]
    assert mine == ref


@pytest.mark.parametrize("case", ["chromset_s0005", "small_full"])
def test_alignments_independent_of_band_ranges(dev, case):
    """Large pairs cut into band ranges on many warps (down to one band per
    range) give the same alignments as whole pairs on one warp each."""
    from distributedpanga_b200.pipeline import alignment_lines
    cs, dig = load_case(case)
    dev.gdb_load(cs)
    dev.index_build(want_entries=False)
    dev.merge(dig["freq_cutoff"])
    got = {}
    try:
        for r in (-1, 1, 64):
            dev.set_ranges(r)
            dev.align()
            got[r] = alignment_lines(*dev.alignments())
    finally:
        dev.set_ranges(0)
    assert len(got[-1]) == dig["aln"]["count"]
    assert got[1] == got[-1]
    assert got[64] == got[-1]


@pytest.mark.parametrize("case", ["chromset_s0005", "many_contigs"])
def test_alignments_independent_of_kernel_build(dev, case):
    """The alignment kernel's builds (two, three or four CTAs per SM), with the
    long-call SM flags off, at 20000 waves, and at 50 waves (nearly every
    SM flagged, so that the flagging warps drain most of the queue), give the
    reference's alignments."""
    import gzip
    import os
    from conftest import GOLDEN
    from distributedpanga_b200.pipeline import alignment_lines
    cs, dig = load_case(case)
    ref = _aln_norm(gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n"))
    dev.gdb_load(cs)
    dev.index_build(want_entries=False)
    dev.merge(dig["freq_cutoff"])
    try:
        for build in (5, 4, 3, 2):
            dev.set_build(build)
            for lw in (0, 50, 20000):
                dev.set_long_waves(lw)
                dev.align()
                assert _aln_norm(alignment_lines(*dev.alignments())) == ref, (build, lw)
    finally:
        dev.set_build(0)
        dev.set_long_waves(-1)


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("case", ["small_s002", "edge_mix"])
def test_1aln_file_matches_reference(dev, case, binary):
    """The GPU path's .1aln file, in either ONE encoding, read by the
    reference's own reader, is the reference's record stream."""
    import gzip
    import os
    import subprocess
    import tempfile
    from conftest import GOLDEN, ROOT
    alndump = os.path.join(ROOT, "oracle", "_ref", "alndump")
    if not os.path.exists(alndump):
        pytest.skip("oracle/_ref not built")
    cs, dig = load_case(case)
    dev.gdb_load(cs)
    dev.index_build(want_entries=False)
    dev.merge(dig["freq_cutoff"])
    dev.align()
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "out.1aln")
        dev.write_1aln(p, db_name="g.1gdb", cwd=d, binary=binary)
        out = subprocess.run([alndump, p], check=True, capture_output=True, text=True).stdout
    mine = [" ".join(l.split()) for l in out.split("\n") if l.strip() and not l.startswith("#")]
    ref = [" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n")
           if l.strip()]
    assert mine == ref


def test_diag_sort_consumes_seeds(dev, oracle):
    """The diagonal sort uses a unit's seed buffer as its second key buffer:
    after it the unit's seeds cannot be copied, sorting the unit again gives
    the same panels without re-sorting, and loading seeds makes it sortable
    again with the same result."""
    from distributedpanga_b200.pipeline import PgaError
    cs, dig = load_case("small_s002")
    dev.gdb_load(cs)
    dev.index_build(want_entries=False)
    dev.merge(dig["freq_cutoff"])
    ns, _ = dev.seeds(0)
    sw, cnt = dev.diag_sort(0)
    a0, o0 = dev.diag_records(0, sw, cnt)
    with pytest.raises(PgaError):
        dev.seeds(0)
    css, _ = dev.seeds(1)                  # the other unit is untouched
    assert (sw, cnt) == dev.diag_sort(0)
    a1, o1 = dev.diag_records(0, sw, cnt)
    assert np.array_equal(a0, a1) and np.array_equal(o0, o1)
    dev.seeds_load(0, ns)
    dev.seeds_load(1, css)
    assert (sw, cnt) == dev.diag_sort(0)
    a2, o2 = dev.diag_records(0, sw, cnt)
    assert np.array_equal(a0, a2) and np.array_equal(o0, o2)
    check_diag(a2, o2, "N", dig)
