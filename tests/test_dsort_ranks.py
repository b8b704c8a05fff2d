"""The distributed index build (distributedpanga_b200.dsort, the reference's
stage 2) on CPU over gloo: ranks holding the records of their own contigs
exchange them by 10-bit bucket, sort locally and fix the seam LCPs; the ranks'
buffers in rank order equal the single-process sorted index byte for byte.
The local sort here is the oracle's (on GPUs it is Device.sort_records)."""
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


def _contig_of(rec: np.ndarray, ctgb: int) -> np.ndarray:
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
    from distributedpanga_b200 import dsort, gdb
    from oracle import binding as orc
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cs, _ = load_case(case)
        posb, ctgb, _ = gdb.record_sizing(cs)
        allrec = orc.extract(cs, posb, ctgb)
        mine = allrec[_contig_of(allrec, ctgb) % world == rank]
        got = dsort.run_stage2(mine, lambda r: orc.sort_records(r))
        out[rank] = got.tobytes()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,world", [("small_s002", 2), ("edge_mix", 3)])
def test_stage2_equals_single_process_index(oracle, case, world):
    from conftest import load_case
    from distributedpanga_b200 import gdb
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, case, out), nprocs=world, start_method="spawn", join=True)
        parts = [out[r] for r in range(world)]
    cs, _ = load_case(case)
    posb, ctgb, rsize = gdb.record_sizing(cs)
    want = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    got = np.frombuffer(b"".join(parts), dtype=np.uint8).reshape(-1, want.shape[1])
    assert sum(len(p) for p in parts) == want.size
    assert all(len(p) > 0 for p in parts)                 # every rank got a share
    assert np.array_equal(got, want)


def _bad_sort_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    from distributedpanga_b200 import dsort
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(rank)
        rec = rng.integers(0, 256, (500, 16)).astype(np.uint8)
        # rank 1's local sort is broken (returns its input unsorted); every
        # rank must learn of it after the same collectives and raise
        sort_fn = (lambda r: r) if rank == 1 else (lambda r: r[np.lexsort(r[:, 10:0:-1].T)])
        try:
            dsort.run_stage2(rec, sort_fn)
            out[rank] = "no error"
        except dsort.Stage2Error as e:
            out[rank] = str(e)
    finally:
        dist.destroy_process_group()


def test_a_failing_rank_fails_every_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_bad_sort_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert all("local sort check failed" in res[r] for r in range(world)), res


def test_destination_map_and_helpers():
    from distributedpanga_b200 import dsort
    rng = np.random.default_rng(5)
    for world in (1, 2, 3, 8, 127):
        counts = rng.integers(0, 50, dsort.NUM_BUCK)
        counts[rng.integers(0, dsort.NUM_BUCK, 200)] = 0
        ksplit, select = dsort.compute_destination_map(counts, world)
        assert ksplit[0] == 0 and ksplit[world] == dsort.NUM_BUCK
        assert select.min() >= 0 and select.max() <= world - 1
        assert np.all(np.diff(select) >= 0)                # contiguous bucket ranges per rank
        loads = np.bincount(select, weights=counts, minlength=world)
        assert loads.sum() == counts.sum()
        if world > 1:
            assert loads.max() <= counts.sum() / world + counts.max() + 1
    # no records at all: every bucket still has a rank
    k, s = dsort.compute_destination_map(np.zeros(dsort.NUM_BUCK, np.int64), 4)
    assert s.min() >= 0 and s.max() <= 3
    x = np.array([0x1b] * 10, np.uint8)
    y = x.copy()
    assert dsort.kmer_lcp_bases(x, y) == 40
    y[3] ^= 0x04                                           # third base of byte 3 differs
    assert dsort.kmer_lcp_bases(x, y) == 14
    rec = np.zeros((3, 16), np.uint8)
    rec[:, 1] = [5, 3, 7]
    assert dsort.verify_per_rank_sorted(rec) == (1, 1)


SPLIT_DUMP = os.path.join(ROOT, "oracle", "_ref", "split_dump")


@pytest.mark.skipif(not os.path.exists(SPLIT_DUMP), reason="oracle/_ref/split_dump not built")
def test_splitter_equals_reference():
    """compute_destination_map equals the reference's (src/dsort.c, compiled
    here) on random global bucket counts -- sparse, skewed, all in one
    bucket, all zero -- at world sizes 1 to 16."""
    import subprocess
    from distributedpanga_b200 import dsort
    rng = np.random.default_rng(9)
    cases = []
    for _ in range(150):
        kind = int(rng.integers(0, 4))
        if kind == 0:
            c = rng.integers(0, 10 ** 6, 1024)
        elif kind == 1:
            c = np.where(rng.random(1024) < 0.9, 0, rng.integers(1, 10 ** 9, 1024))
        elif kind == 2:
            c = (10 ** rng.uniform(0, 9, 1024)).astype(np.int64)
        else:
            c = np.zeros(1024, np.int64)
            c[int(rng.integers(0, 1024))] = int(rng.integers(1, 10 ** 6))
        cases.append(c)
    cases.append(np.zeros(1024, np.int64))
    for c in cases:
        world = int(rng.integers(1, 17))
        out = subprocess.run([SPLIT_DUMP], input="%d\n%s\n" % (world, " ".join(str(int(v)) for v in c)),
                             capture_output=True, text=True, check=True).stdout.split("\n")
        ksplit, select = dsort.compute_destination_map(np.asarray(c, np.int64), world)
        assert list(ksplit) == [int(v) for v in out[0].split()]
        assert list(select) == [int(v) for v in out[1].split()]
        # the reference's S-08 invariants: select non-decreasing and in range,
        # ksplit non-decreasing and ending at the bucket count
        sel = np.asarray(select)
        assert np.all(np.diff(sel) >= 0) and sel.min() >= 0 and sel.max() < world
        assert np.all(np.diff(np.asarray(ksplit)) >= 0) and ksplit[world] == 1024
    ksplit, select = dsort.compute_destination_map(np.full(1024, 7, np.int64), 4)
    assert list(select) == [b // 256 for b in range(1024)]


def _seam_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    from distributedpanga_b200 import dsort
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rec = _seam_records()
        counts = dsort.bucket_local_counts(rec)
        _, select = dsort.compute_destination_map(counts, world)

        def sort_fn(r):
            r = r[np.lexsort(r[:, 10:0:-1].T)].copy()
            r[0, 0] = 0
            for i in range(1, len(r)):
                r[i, 0] = dsort.kmer_lcp_bases(r[i - 1, 1:11], r[i, 1:11])
            return r

        got = dsort.run_stage2(rec[rank::world], sort_fn)
        out[rank] = (got.tobytes(), [int(select[768]), int(select[769]), int(select[770])])
    finally:
        dist.destroy_process_group()


def _seam_records():
    """The reference's R-01 fixture: every k-mer's first byte 0xC0, four
    records in bucket 768 (second byte's top bits 00) and four in bucket 770
    (10), distinct in bytes 2..9; bucket 769 empty."""
    rng = np.random.default_rng(21)
    rec = np.zeros((8, 16), np.uint8)
    rec[:, 1] = 0xC0
    rec[:4, 2] = 0x00
    rec[4:, 2] = 0x80
    rec[:, 3:11] = rng.integers(0, 256, (8, 8))
    rec[:, 11:] = np.arange(8)[:, None]
    return rec


def test_r01_seam_lcp_past_an_empty_rank():
    """World 4: the splitter sends bucket 768 to rank 0, the empty 769 to
    rank 1 and 770 to rank 2, so rank 1 holds nothing and rank 2's first
    record takes its LCP from rank 0's last k-mer: 4 bases (the first byte
    and nothing of the second).  The ranks' slices in order are the sorted
    index with its LCPs."""
    from distributedpanga_b200 import dsort
    world = 4
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_seam_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = {r: out[r] for r in range(world)}
    assert res[0][1] == [0, 1, 2]
    parts = [np.frombuffer(res[r][0], np.uint8).reshape(-1, 16) for r in range(world)]
    assert [len(p) for p in parts] == [4, 0, 4, 0]
    assert parts[2][0, 0] == 4
    rec = _seam_records()
    want = rec[np.lexsort(rec[:, 10:0:-1].T)].copy()
    want[0, 0] = 0
    for i in range(1, 8):
        want[i, 0] = dsort.kmer_lcp_bases(want[i - 1, 1:11], want[i, 1:11])
    assert np.array_equal(np.concatenate(parts), want)
