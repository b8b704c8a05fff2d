"""Seeds to their contig pair's owner (distributedpanga_b200.seed_exchange,
the reference's stage 3 routing) on CPU over gloo: after the distributed
index build each rank merges its own bucket range (the oracle's k-mer table
and adaptamer merge here; the device drop-ins on GPUs) and routes its seeds;
each rank then holds exactly the single-process seeds of the pairs it owns,
and its diagonal sort gives the single-process panels restricted to those
pairs, in the same order."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


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
    from distributedpanga_b200 import dsort, gdb, seed_exchange as sx
    from oracle import binding as orc
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cs, dig = load_case(case)
        posb, ctgb, _ = gdb.record_sizing(cs)
        allrec = orc.extract(cs, posb, ctgb)
        mine = dsort.run_stage2(allrec[_contig_of(allrec, ctgb) % world == rank], orc.sort_records)
        ent, cum, _ = orc.build_adapter(mine, posb, ctgb)
        ns, css, _, _ = orc.merge(ent, cum, posb, ctgb, dig["freq_cutoff"], cs.ncontig)
        owner, _ = sx.contig_assignment_build(cs.clen, world)
        rfp = sx.rank_for_pair(owner)
        rn = sx.redistribute_seeds(ns, posb, ctgb, rfp)
        rc = sx.redistribute_seeds(css, posb, ctgb, rfp)
        # each rank's diagonal sort of what it received
        dbyte, _ = gdb.diag_sizing(cs, ctgb)
        panels = [orc.reimport_sort(u, posb, ctgb, comp, cs.ncontig, cs.maxctg, dbyte)
                  for comp, u in ((0, rn), (1, rc))]
        out[rank] = (rn.tobytes(), rc.tobytes(), [(a.tobytes(), o.tolist()) for a, o in panels])
    finally:
        dist.destroy_process_group()


def _rows(a):
    return a[np.lexsort(a.T[::-1])] if len(a) else a


@pytest.mark.parametrize("case,world", [("small_s002", 2), ("many_contigs", 3)])
def test_each_rank_gets_the_seeds_of_its_pairs(oracle, case, world):
    from conftest import load_case
    from distributedpanga_b200 import gdb, seed_exchange as sx
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, case, out), nprocs=world, start_method="spawn", join=True)
        res = {r: out[r] for r in range(world)}
    cs, dig = load_case(case)
    posb, ctgb, _ = gdb.record_sizing(cs)
    sb = 1 + 2 * (posb + ctgb)
    ent, cum, _ = oracle.build_adapter(oracle.sort_records(oracle.extract(cs, posb, ctgb)), posb, ctgb)
    ns, css, _, _ = oracle.merge(ent, cum, posb, ctgb, dig["freq_cutoff"], cs.ncontig)
    rfp = sx.rank_for_pair(sx.contig_assignment_build(cs.clen, world)[0])
    total = [0, 0]
    for unit, allseeds in ((0, ns), (1, css)):
        a, b = sx.seed_contigs(allseeds, posb, ctgb)
        for r in range(world):
            got = np.frombuffer(res[r][unit], dtype=np.uint8).reshape(-1, sb)
            want = allseeds[rfp[a, b] == r]
            assert np.array_equal(_rows(got), _rows(want)), (unit, r)
            total[unit] += len(got)
    assert total == [len(ns), len(css)] and total[0] > 0
    # the ranks' diagonal-sorted panels are the single-process panels, each
    # restricted to the pairs the rank owns, in the same order
    dbyte, _ = gdb.diag_sizing(cs, ctgb)
    for unit, allseeds in ((0, ns), (1, css)):
        arr, off = oracle.reimport_sort(allseeds, posb, ctgb, unit, cs.ncontig, cs.maxctg, dbyte)
        sw = arr.shape[1] if arr.ndim == 2 else 0
        if len(arr) == 0:
            continue
        j = np.zeros(len(arr), dtype=np.int64)
        for bb in range(ctgb):
            j |= arr[:, sw - ctgb + bb].astype(np.int64) << (8 * bb)
        j &= (1 << (8 * ctgb - 1)) - 1
        a_of = np.repeat(np.arange(cs.ncontig), np.diff(np.asarray(off)))
        for r in range(world):
            got, goff = res[r][2][unit]
            got = np.frombuffer(got, dtype=np.uint8).reshape(-1, sw)
            keep = rfp[a_of, j] == r
            assert np.array_equal(got, arr[keep]), (unit, r)
            want_off = np.concatenate([[0], np.cumsum(np.bincount(a_of[keep], minlength=cs.ncontig))])
            assert np.array_equal(np.asarray(goff), want_off), (unit, r)


def test_assignment_and_plan():
    from distributedpanga_b200 import seed_exchange as sx
    clen = [500, 300, 300, 100, 50]
    owner, load = sx.contig_assignment_build(clen, 2)
    # the heaviest pair (0, 0) goes to rank 0, the next (0, 1) to rank 1, ...
    assert owner[0, 0] == 0 and owner[0, 1] == 1
    assert (owner[np.tril_indices(5, -1)] == -1).all() and (owner[np.triu_indices(5)] >= 0).all()
    assert load.sum() == sum(clen[i] * clen[j] for i in range(5) for j in range(i, 5))
    rfp = sx.rank_for_pair(owner)
    assert (rfp == rfp.T).all() and (rfp >= 0).all()
    assert sx.plan_byte_exchange([3, 0, 5]) == ([3, 0, 5], [0, 3, 3])
    assert sx.plan_byte_exchange([-1]) == -1
    assert sx.plan_byte_exchange([2 ** 31]) == -2
    assert sx.plan_byte_exchange([2 ** 30, 2 ** 30]) == -3
    with pytest.raises(ValueError):
        sx.contig_assignment_build(clen, 128)


ASSIGN_DUMP = os.path.join(ROOT, "oracle", "_ref", "assign_dump")


@pytest.mark.skipif(not os.path.exists(ASSIGN_DUMP), reason="oracle/_ref/assign_dump not built")
def test_assignment_equals_reference():
    """contig_assignment_build equals the reference's own (src/contig_assignment.c,
    compiled here) on random contig sets with many equal lengths (ties in
    weight and in load decide by pair and by rank) at world sizes 1 to 9."""
    import subprocess
    from distributedpanga_b200 import seed_exchange as sx
    rng = np.random.default_rng(5)
    for _ in range(120):
        n = int(rng.integers(1, 45))
        world = int(rng.integers(1, 10))
        clen = rng.choice(rng.integers(1, 3000, int(rng.integers(1, 6))), n)
        txt = "%d %d\n%s\n" % (n, world, " ".join(str(int(c)) for c in clen))
        out = subprocess.run([ASSIGN_DUMP], input=txt, capture_output=True, text=True, check=True).stdout.split("\n")
        ref_owner = np.array([[int(v) for v in l.split()] for l in out[:n]], dtype=np.int8)
        ref_load = np.array([int(v) for v in out[n].split()], dtype=np.int64)
        owner, load = sx.contig_assignment_build(clen, world)
        assert np.array_equal(owner, ref_owner)
        assert np.array_equal(load, ref_load)
