"""The served form on the GPU: a request against a resident target gives, bit
for bit, what the plain path gives on the GDB of the target's text followed
by the query's -- the GDB tables, the sorted index and its k-mer table
entries, and the alignments -- and the same alone and in a mix of
concurrent requests."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_target(dev):
    from distributedpanga_b200 import pipeline, synth
    contigs = synth.make_target(scale=0.002)
    text = synth.fasta_bytes(contigs, "t")
    t = pipeline.Target(text)
    yield contigs, text, t
    t.close()


def _same_tables(a, b):
    assert np.array_equal(a.bps, b.bps)
    assert np.array_equal(a.contigs, b.contigs)
    assert np.array_equal(a.scaffolds, b.scaffolds)
    assert a.headers == b.headers
    assert np.array_equal(a.count, b.count) and a.maxctg == b.maxctg


def _check_request(dev_s, dev_p, target, ttext, qtext):
    ts = dev_s.serve_load(target, qtext, want_entries=True, tables=True)
    tp = dev_p.gdb_ingest_fasta(ttext + qtext)
    _same_tables(ts, tp)
    assert dev_p.index_build(want_entries=True) == dev_s.nrec
    assert dev_s.record_sizing() == dev_p.record_sizing()
    assert np.array_equal(dev_s.index_records(), dev_p.index_records())
    es, cs, bs = dev_s.index_entries()
    ep, cp, bp = dev_p.index_entries()
    assert np.array_equal(es, ep) and np.array_equal(cs, cp) and bs == bp


def test_serve_load_index_equals_plain(dev, small_target):
    from distributedpanga_b200 import pipeline, synth
    contigs, ttext, target = small_target
    assert target.ncontig == len(contigs) and target.bases == sum(len(c) for c in contigs)
    dp = pipeline.Device(0)
    try:
        for k, (_, q) in enumerate(synth.query_stream(contigs, 3, 0.0, 20_000, 300_000, seed=21, median=60_000)):
            _check_request(dev, dp, target, ttext, synth.fasta_bytes(q, "q%d_" % k))
    finally:
        dp.close()


def test_serve_load_edge_queries(dev):
    """A query that widens the contig|strand field (the target's records are
    re-encoded in the union), one with no k-mers at all, one with N runs
    and lower case, and a rejected query that leaves the context usable."""
    from distributedpanga_b200 import pipeline, synth
    rng = np.random.default_rng(41)
    tcontigs = [rng.integers(0, 4, int(n)).astype(np.uint8) for n in rng.integers(2_000, 9_000, 100)]
    ttext = synth.fasta_bytes(tcontigs, "t")
    target = pipeline.Target(ttext)
    dp = pipeline.Device(0)
    try:
        wide = [c[100:1500] for c in tcontigs[:40]]                  # 140 contigs: 2-byte contig field
        _check_request(dev, dp, target, ttext, synth.fasta_bytes(wide, "w"))
        assert dev.record_sizing()[1] == 2
        _check_request(dev, dp, target, ttext, b">tiny\nACGTA\n>tiny2\nGG\n")
        mixed = b">m1 with spaces\nacgtNNNNNNNNNNacgtacgtTTGACCA\n" + synth.fasta_bytes([tcontigs[3][:777]], "m")
        _check_request(dev, dp, target, ttext, mixed)
        with pytest.raises(pipeline.PgaError):
            dev.serve_load(target, b">bad\n")
        _check_request(dev, dp, target, ttext, synth.fasta_bytes([tcontigs[7]], "again"))
    finally:
        dp.close()
        target.close()


def test_served_mix_equals_plain_alone(small_target):
    """Four requests admitted together on two slots: each one's alignments
    are the plain path's for that request run alone."""
    from distributedpanga_b200 import pipeline, serve, synth
    contigs, ttext, target = small_target
    stream = synth.query_stream(contigs, 4, 0.0, 30_000, 400_000, seed=22, median=80_000)
    reqs = []
    for k, (arr, q) in enumerate(stream):
        text = synth.fasta_bytes(q, "q%d_" % k)
        reqs.append(serve.Request(k, text, 0.0, sum(len(c) for c in q)))
    srv = serve.Server(target, slots=2)
    try:
        res, summary = srv.run(reqs)
    finally:
        srv.close()
    assert summary["requests"] == 4 and summary["p99_latency_s"] >= summary["p50_latency_s"] > 0
    assert len({r.slot for r in res}) == 2
    dp = pipeline.Device(0)
    try:
        for r, q in zip(res, reqs):
            p = serve.plain_request(dp, ttext, q.text)
            assert r.out["nalign"] == p["nalign"] > 0
            assert r.out["records"] == p["records"]
            for a, b in zip(r.out["alignments"], p["alignments"]):
                assert np.array_equal(a, b)
    finally:
        dp.close()


def test_served_call_record_equals_plain(dev):
    """A target with the record of its own Local_Alignment calls: a request's
    calls on two target contigs with recorded inputs take the recorded
    results, and every request's alignments are still, bit for bit, the
    plain path's -- also for a query contig longer than the target's longest
    (every diagonal value of the key layout moves; the calls' inputs do
    not)."""
    from distributedpanga_b200 import pipeline, serve, synth
    contigs = synth.make_target(scale=0.005)
    ttext = synth.fasta_bytes(contigs, "t")
    target = pipeline.Target(ttext, reuse=True)
    dp = pipeline.Device(0)
    try:
        queries = [q for _, q in synth.query_stream(contigs, 3, 0.0, 20_000, 600_000, seed=23, median=100_000)]
        longest = max(range(len(contigs)), key=lambda i: len(contigs[i]))
        other = (longest + 1) % len(contigs)
        queries.append([np.concatenate([contigs[longest], contigs[other]])])
        for k, q in enumerate(queries):
            qtext = synth.fasta_bytes(q, "q%d_" % k)
            dev.serve_load(target, qtext)
            dev.merge(10)
            n = dev.align()
            st = dev.reuse_stats()
            got = dev.alignments()
            p = serve.plain_request(dp, ttext, qtext)
            assert n == p["nalign"] > 0
            for a, b in zip(got, p["alignments"]):
                assert np.array_equal(a, b)
            assert st["used"] and st["not_used"] is None
            assert 0 < st["calls_from_record"] <= st["calls"]
    finally:
        dp.close()
        target.close()
