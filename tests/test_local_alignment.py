"""pga_local_alignment: Local_Alignment on request lists equals the
reference's own Local_Alignment (lib/align.c:1423, compiled from its sources
into oracle/_ref/la_batch) on the same contigs: paths and trace values."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT

LA_BATCH = os.path.join(ROOT, "oracle", "_ref", "la_batch")
FA2GDB = os.path.join(ROOT, "oracle", "_ref", "fa2gdb")


def contigs_and_requests(seed=11):
    from distributedpanga_b200 import synth
    rng = np.random.default_rng(seed)
    a = synth.random_bases(rng, 30000, 0.45)
    b = synth.indels(rng, synth.substitute(rng, a, 0.03), 0.004, lambda k: rng.integers(1, 6, size=k), 0.45)
    c = synth.revcomp(synth.substitute(rng, a[6000:18000], 0.02))
    d = synth.random_bases(rng, 5000, 0.5)
    contigs = [a, b, c, d]
    req = []
    for p in range(500, 29000, 1500):          # a against its diverged copy, along diagonal ~0
        req.append([0, 1, 0, -25, 25, 2 * p, -1, -1])
    for p in range(1000, 11000, 2000):         # the reverse-complemented segment: diagonal -6000
        req.append([2, 0, 1, -6020, -5980, 2 * p + 6000, -1, -1])
    for p in range(2000, 28000, 4000):         # self hits constrained to one side of diagonal 0
        req.append([0, 0, 0, 5, 40, 2 * p + 20, 4, -1])
    for _ in range(16):                        # random bands inside the contigs: mostly nothing to align
        i, j = int(rng.integers(0, 4)), int(rng.integers(0, 4))
        la, lb = len(contigs[i]), len(contigs[j])
        w = int(rng.integers(0, 60))
        x0, y0 = int(rng.integers(w + 1, la - w - 1)), int(rng.integers(w + 1, lb - w - 1))
        req.append([i, j, int(rng.integers(0, 2)), x0 - y0 - w, x0 - y0, x0 + y0, -1, -1])
    return contigs, np.array(req, dtype=np.int32)


def reference_paths(contigs, req):
    from distributedpanga_b200 import synth
    with tempfile.TemporaryDirectory() as d:
        fa = os.path.join(d, "g.fa")
        synth.write_fasta(fa, contigs)
        subprocess.run([FA2GDB, fa, os.path.join(d, "g.1gdb")], check=True, capture_output=True)
        rq = os.path.join(d, "req.txt")
        np.savetxt(rq, req, fmt="%d")
        out = subprocess.run([LA_BATCH, os.path.join(d, "g"), rq], check=True, capture_output=True,
                             text=True).stdout
    rows = []
    for line in out.strip().split("\n"):
        head, tr = line.split(";")
        rows.append(([int(x) for x in head.split()], [int(x) for x in tr.split()]))
    return rows


@pytest.mark.gpu
def test_local_alignment_matches_reference(dev):
    if not os.path.exists(LA_BATCH):
        pytest.skip("oracle/_ref not built")
    from distributedpanga_b200 import gdb
    contigs, req = contigs_and_requests()
    ref = reference_paths(contigs, req)
    cs = gdb.from_contigs(contigs)
    dev.gdb_load(cs)
    dev.set_freq(cs.freq)
    path, toff, tr = dev.local_alignment(req)
    assert (path[:, 6] == 0).all()
    long_ones = 0
    for i, (head, rtr) in enumerate(ref):
        assert path[i, :6].tolist() == head, (i, req[i].tolist(), path[i].tolist(), head)
        assert tr[toff[i]:toff[i + 1]].tolist() == rtr, i
        long_ones += head[1] - head[0] > 1000
    assert long_ones >= 10      # the band requests found real alignments


@pytest.mark.gpu
def test_local_alignment_rejects_bad_requests(dev):
    from distributedpanga_b200 import gdb, pipeline
    contigs, req = contigs_and_requests()
    dev.gdb_load(gdb.from_contigs(contigs))
    bad = req[:1].copy()
    bad[0, 0] = 7                               # no such contig
    with pytest.raises(pipeline.PgaError):
        dev.local_alignment(bad)
    bad = req[:1].copy()
    bad[0, 3], bad[0, 4] = 10, 5                # low > hgh
    with pytest.raises(pipeline.PgaError):
        dev.local_alignment(bad)
    bad = req[:1].copy()
    bad[0, 5] = 5                               # starts before the contigs
    with pytest.raises(pipeline.PgaError):
        dev.local_alignment(bad)
