"""FastGA's self-pair order across ranks (distributedpanga_b200.sharded_order).

On CPU over gloo: the sharded index build, the seed routing by pair owner,
each rank aligning the pairs it owns with the host aligner (align_core.cuh,
the code the GPU kernel's chain driver shares), and the order values combined
with all-reduce(MAX).  The union of the ranks' alignments must be the
reference's .1aln record stream of the single-process run, and every rank
must decide the same entry value for every self pair."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import GOLDEN, ROOT
from test_align_host import aht  # noqa: F401  (the host aligner fixture)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _contig_of(rec, ctgb):
    v = np.zeros(len(rec), dtype=np.int64)
    for b in range(ctgb):
        v |= rec[:, rec.shape[1] - ctgb + b].astype(np.int64) << (8 * b)
    return v & ((1 << (8 * ctgb - 1)) - 1)


def _worker(rank, world, port, case, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_case
    from test_align_host import aln_lines, load_aht, run_unit
    from distributedpanga_b200 import dsort, seed_exchange as sx, sharded_order as so
    from oracle import binding as orc
    dist.init_process_group("gloo", rank=rank, world_size=world)

    def allreduce(a, op):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64))
        dist.all_reduce(t, op=op)
        return t.numpy()

    try:
        aht = load_aht()
        cs, dig = load_case(case)
        n, posb, ctgb = cs.ncontig, dig["posb"], dig["ctgb"]
        allrec = orc.extract(cs, posb, ctgb)
        mine = dsort.run_stage2(allrec[_contig_of(allrec, ctgb) % world == rank], orc.sort_records)
        ent, cum, _ = orc.build_adapter(mine, posb, ctgb)
        ns, css, nb, _ = orc.merge(ent, cum, posb, ctgb, dig["freq_cutoff"], n)
        rfp = sx.rank_for_pair(sx.contig_assignment_build(cs.clen, world)[0])
        rn = sx.redistribute_seeds(ns, posb, ctgb, rfp)
        rc = sx.redistribute_seeds(css, posb, ctgb, rfp)
        arrN, offN = orc.reimport_sort(rn, posb, ctgb, 0, n, cs.maxctg, dig["dbyte"])
        arrC, offC = orc.reimport_sort(rc, posb, ctgb, 1, n, cs.maxctg, dig["dbyte"])
        nb = allreduce(nb, dist.ReduceOp.SUM)

        perm, pos = so.order_positions(cs.clen)
        rs = so.range_starts(cs.clen, nb, dig["swide"], perm)
        # first pass: every pair this rank owns; those of two contigs are final
        _, pairsN = run_unit(aht, cs, arrN, offN, dig, 0)
        lk, eb = so.local_keys(pairsN, pos, n)
        st = np.zeros(n, dtype=np.int64)
        for a, b, _, _ in pairsN:
            if a == b:
                st[pos[a]] = 1
        lk, eb, st = (allreduce(v, dist.ReduceOp.MAX) for v in (lk, eb, st))

        entry = np.zeros(n, dtype=np.int32)
        aligned = []

        def align_round(new):
            for c, v in new.items():
                entry[c] = v
            own = [c for c in new if rfp[c, c] == rank]
            if not own:
                return {}
            _, pr = run_unit(aht, cs, arrN, offN, dig, 0, entry)
            res = {(int(a), int(b)): (int(k), int(e)) for a, b, k, e in pr}
            aligned.extend(own)
            return {c: res[(c, c)] for c in own}

        values, rounds = so.resolve(n, pos, rs, lk, eb, st, align_round,
                                    lambda a: allreduce(a, dist.ReduceOp.MAX))
        outN, _ = run_unit(aht, cs, arrN, offN, dig, 0, entry)
        outC, _ = run_unit(aht, cs, arrC, offC, dig, 1)
        out[rank] = (aln_lines(outN + outC), sorted(values.items()), rounds, sorted(aligned),
                     int((st == 1).sum()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,world,nself", [("small_s002", 2, 6), ("small_s002", 3, 6), ("chromset_s0005", 3, 2),
                                              ("many_contigs", 3, 0)])
def test_ranks_alignments_are_the_single_process_stream(oracle, aht, case, world, nself):
    import gzip
    from conftest import load_case
    from distributedpanga_b200 import seed_exchange as sx
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, case, out), nprocs=world, start_method="spawn", join=True)
        res = {r: out[r] for r in range(world)}
    cs, dig = load_case(case)
    ref = sorted(" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read()
                 .split("\n") if l.strip())
    mine = sorted(" ".join(l.split()) for r in range(world) for l in res[r][0])
    assert len(mine) == dig["aln"]["count"]
    assert mine == ref
    # every rank decided the same values in the same number of rounds, each
    # self pair was aligned by its owner alone, and every one of them got a value
    assert all(res[r][1] == res[0][1] and res[r][2] == res[0][2] for r in range(world))
    assert res[0][4] == len(res[0][1]) == nself
    rfp = sx.rank_for_pair(sx.contig_assignment_build(cs.clen, world)[0])
    got = sorted(c for r in range(world) for c in res[r][3])
    assert got == sorted(c for c, _ in res[0][1])
    assert all(rfp[c, c] == r for r in range(world) for c in res[r][3])
    if nself > 2:
        assert sum(1 for r in range(world) if res[r][3]) >= 2


def _fake_round(outcomes, log):
    """align_round of one rank that owns every self pair: outcomes[c] =
    (calls, exit bepos) whatever the entry value."""
    def run(new):
        log.append(dict(new))
        return {c: outcomes[c] for c in new if c in outcomes}
    return run


def test_resolve_rows_and_waits():
    from distributedpanga_b200 import sharded_order as so
    # contigs 0..4 in order 0..4 (lengths decreasing), one range [0, 5)
    pos, rs, n = np.arange(5), [0] * 5, 5
    lk = np.zeros(n, dtype=np.int64)
    eb = np.zeros(n, dtype=np.int64)
    st = np.array([0, 1, 0, 1, 1], dtype=np.int64)
    # row 2 has a later partner (position 4) that called: its exit bepos 77
    lk[2] = (5 << 32) | 77
    log = []
    vals, rounds = so.resolve(n, pos, rs, lk, eb, st, _fake_round({1: (3, 41), 3: (0, 0), 4: (2, 9)}, log),
                              lambda a: a)
    # 1: nothing earlier in the first range (the unset value); 3: row 2's
    # later partner; 4: waits for 3, which made no call, then row 2 again
    assert vals == {1: so.UNSET_MAIN, 3: 77, 4: 77}
    assert rounds == 2 and log == [{1: so.UNSET_MAIN, 3: 77}, {4: 77}]
    # the same self pairs in a range that starts at 1: position 1 opens it (0)
    vals, _ = so.resolve(n, pos, [0, 1, 1, 1, 1], lk, eb, st, _fake_round({1: (3, 41), 3: (0, 0), 4: (2, 9)}, []),
                         lambda a: a)
    assert vals == {1: 0, 3: 77, 4: 77}
    # without row 2's call, 3 takes 1's exit bepos, and 4 then takes 3's
    lk[2] = 0
    vals, rounds = so.resolve(n, pos, rs, lk, eb, st, _fake_round({1: (3, 41), 3: (1, 12), 4: (2, 9)}, []),
                              lambda a: a)
    assert vals == {1: so.UNSET_MAIN, 3: 41, 4: 12} and rounds == 3
    # an earlier partner that called decides at once
    eb[4] = (2 << 32) | 5
    vals, rounds = so.resolve(n, pos, rs, lk, eb, st, _fake_round({1: (3, 41), 3: (1, 12), 4: (2, 9)}, []),
                              lambda a: a)
    assert vals == {1: so.UNSET_MAIN, 3: 41, 4: 5} and rounds == 2
    # a self pair that no rank reports stays pending: an error on every rank
    with pytest.raises(RuntimeError):
        so.resolve(n, pos, rs, lk, eb, st, _fake_round({1: (3, 41), 4: (2, 9)}, []), lambda a: a)


def test_range_starts_and_keys():
    from distributedpanga_b200 import sharded_order as so
    perm, pos = so.order_positions([5, 9, 9, 1])
    assert perm.tolist() == [1, 2, 0, 3] and pos.tolist() == [2, 0, 1, 3]
    # four contigs of one part; seeds split into ranges of about 1/32 of the part
    rs = so.range_starts([5, 9, 9, 1], [0, 10, 0, 0], 1, perm)
    assert rs == [0, 1, 2, 3]
    lk, eb = so.local_keys([(0, 1, 2, 30), (0, 3, 1, 40), (0, 0, 5, 1), (2, 0, 0, 7)], pos, 4)
    # anchor 0 at position 2: partner 1 (position 0, earlier) and 3 (position 3, later)
    assert lk.tolist() == [0, 0, (4 << 32) | 40, 0]
    assert eb.tolist() == [0, 0, (1 << 32) | 30, 0]


def _fastga_loop(n, rs, partners, self_pairs, pair_out, self_out):
    """Entry values by FastGA's own loop: in each range, rows in order, each
    row's partners in order with the self pair at its own position, the last
    Local_Alignment call's exit bepos carried along (the unset value at a
    range start).  Contig c sits at order position c."""
    entry = {}
    last = None
    for x in range(n):
        if rs[x] == x:
            last = 32767 if x == 0 else 0
        for b in sorted(partners[x] | ({x} if x in self_pairs else set())):
            if b == x:
                entry[x] = last
                calls, bep = self_out(x, last)
            else:
                calls, bep = pair_out[(x, b)]
            if calls > 0:
                last = bep
    return entry


@pytest.mark.parametrize("seed", range(40))
def test_resolve_equals_fastga_loop(seed):
    """Random orders, ranges, pair outcomes and self pairs whose outcome
    depends on their entry value: the values resolve() decides are those of
    FastGA's sequential loop, alone and with the self pairs owned by three
    ranks that combine their states with all-reduce(MAX) (threads here)."""
    import threading
    from distributedpanga_b200 import sharded_order as so
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 40))
    cuts = sorted(set([0] + rng.integers(1, max(2, n), int(rng.integers(0, 5))).tolist()))
    rs = [max(c for c in cuts if c <= x) for x in range(n)]
    partners = [set(int(b) for b in rng.choice(n, int(rng.integers(0, min(n, 6))), replace=False)) - {x}
                for x in range(n)]
    pair_out = {(x, b): (int(rng.random() < 0.5), int(rng.integers(0, 5000))) for x in range(n) for b in partners[x]}
    self_pairs = set(int(x) for x in np.nonzero(rng.random(n) < 0.6)[0])
    salt = int(rng.integers(1, 1000))

    def self_out(x, entry):
        return int((entry + salt + x) % 3 != 0), (entry * 7 + salt + x) % 4000

    want = _fastga_loop(n, rs, partners, self_pairs, pair_out, self_out)
    pos = np.arange(n)
    lk, eb = so.local_keys([(x, b, c, e) for (x, b), (c, e) in pair_out.items()], pos, n)
    st = np.zeros(n, dtype=np.int64)
    st[list(self_pairs)] = 1

    got, _ = so.resolve(n, pos, rs, lk, eb, st, lambda new: {c: self_out(c, v) for c, v in new.items()},
                        lambda a: a)
    assert got == want

    world = 3
    vals, cells = [None] * world, [None] * world
    bar = threading.Barrier(world)

    def allreduce_max(r, a):
        cells[r] = np.array(a)
        bar.wait()
        out = np.max(np.stack(cells), axis=0)
        bar.wait()
        return out

    def rank(r):
        own = lambda new: {c: self_out(c, v) for c, v in new.items() if c % world == r}
        vals[r] = so.resolve(n, pos, rs, lk, eb, st, own, lambda a: allreduce_max(r, a))[0]

    ts = [threading.Thread(target=rank, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert all(v == want for v in vals)


FO_CORE = os.path.join(ROOT, "oracle", "_ref", "libfo_core.so")
needs_fo = pytest.mark.skipif(not os.path.exists(FO_CORE), reason="oracle/_ref/libfo_core.so not built")


def _fo_core():
    """The reference's own rules (src/fastga_order_core.c, compiled into
    oracle/_ref by oracle/Makefile)."""
    import ctypes as C
    L = C.CDLL(FO_CORE)
    vp, ci, i64 = C.c_void_p, C.c_int, C.c_int64
    L.fo_compute_ranges.argtypes = [ci, vp, i64, vp, i64, ci, vp, vp, vp, vp]
    L.fo_compute_ranges.restype = ci
    L.fo_from_rows.argtypes = [vp, vp, ci, ci, ci, vp, vp, vp]
    L.fo_from_rows.restype = ci
    L.fo_from_answers.argtypes = [vp, ci, ci, ci, ci, vp, vp]
    L.fo_from_answers.restype = ci
    return L


@needs_fo
def test_range_starts_equal_reference():
    """range_starts -- the GPU path's own rule (pga_fastga_ranges, the host
    code pga_align uses) -- equals the reference's fo_compute_ranges on
    random contig sets (lengths over five decades, contigs without seeds, 1
    to 32 threads)."""
    import ctypes as C
    from distributedpanga_b200 import sharded_order as so
    L = _fo_core()
    rng = np.random.default_rng(11)
    for _ in range(300):
        n = int(rng.integers(1, 300))
        clen = (10 ** rng.uniform(2, 7, n)).astype(np.int64)
        seeds = np.where(rng.random(n) < 0.3, 0, rng.integers(1, 10 ** 5, n)).astype(np.int64)
        swide, T = int(rng.integers(9, 15)), int(rng.choice([1, 2, 7, 32]))
        perm, _ = so.order_positions(clen)
        cp = np.ascontiguousarray(clen[perm])
        sp = np.ascontiguousarray(seeds[perm])
        rs = np.zeros(n, dtype=np.int32)
        nparts = C.c_int()
        L.fo_compute_ranges(n, cp.ctypes.data, int(clen.sum()), sp.ctypes.data, swide, T, rs.ctypes.data, None,
                            None, C.byref(nparts))
        assert so.range_starts(clen, seeds, swide, perm, T) == rs.tolist()


@needs_fo
def test_row_and_partner_rules_equal_reference():
    """from_rows equals fo_from_rows, and the values first_values decides
    before any self pair runs equal fo_from_answers with every answer in
    (bepos 0 a real value), on random rows, states and partners."""
    import ctypes as C
    from distributedpanga_b200 import sharded_order as so
    L = _fo_core()
    rng = np.random.default_rng(12)
    bep, row, frm, k = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    for _ in range(3000):
        n = int(rng.integers(1, 30))
        x = int(rng.integers(0, n))
        rs = [0] * n
        rs[x] = int(rng.integers(0, x + 1))
        lk = np.zeros(n, dtype=np.int64)
        st = np.zeros(n, dtype=np.int64)
        for y in range(n):
            if rng.random() < 0.5:
                b = int(rng.integers(0, n))
                if b != y:
                    lk[y] = ((b + 1) << 32) | int(rng.choice([0, int(rng.integers(0, 5000))]))
            st[y] = int(rng.choice([0, 1, 2, 3, 3 + int(rng.integers(0, 5000))]))
        rc = L.fo_from_rows(lk.ctypes.data, st.ctypes.data, x, rs[x], so.UNSET_MAIN, C.byref(bep), C.byref(row),
                            C.byref(frm))
        val, wait = so.from_rows(x, lk, st, rs)
        assert wait == (rc == 0)
        if rc == 1:
            assert (val is None) == (row.value == -1)
            assert (val if val is not None else (so.UNSET_MAIN if rs[x] == 0 else 0)) == bep.value
        # the earlier partners of x, nearest first, each with its outcome
        near = sorted(set(int(b) for b in rng.integers(0, x + 1, int(rng.integers(0, 6)))) - {x}, reverse=True)
        out = [(int(rng.random() < 0.5), int(rng.choice([0, int(rng.integers(0, 5000))]))) for _ in near]
        answers = np.array([e if c else -2 for c, e in out] or [0], dtype=np.int32)
        eb = np.zeros(n, dtype=np.int64)
        for b, (c, e) in zip(near, out):
            if c:
                eb[x] = max(eb[x], ((b + 1) << 32) | e)
        s1 = np.zeros(n, dtype=np.int64)
        s1[x] = 1
        rc = L.fo_from_answers(answers.ctypes.data, len(near), x, rs[x], so.UNSET_MAIN, C.byref(bep), C.byref(k))
        known = so.first_values(s1, eb, rs)
        assert (x in known) == (rc == 1)
        if rc == 1:
            assert known[x] == bep.value


@pytest.mark.parametrize("k", range(1, 13))
def test_dependent_chain_takes_k_rounds(k):
    """A chain of k self pairs, each taking its value from the one before it
    (one range, no partners), resolves in exactly k rounds."""
    from distributedpanga_b200 import sharded_order as so
    pos = np.arange(k)
    st = np.ones(k, dtype=np.int64)
    zero = np.zeros(k, dtype=np.int64)
    vals, rounds = so.resolve(k, pos, [0] * k, zero, zero, st, lambda new: {c: (1, v + 1 if c else 5)
                                                                             for c, v in new.items()}, lambda a: a)
    assert rounds == k
    assert vals == {c: (so.UNSET_MAIN if c == 0 else 5 + c - 1) for c in range(k)}
