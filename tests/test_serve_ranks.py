"""The served form on several ranks, on CPU over gloo: each rank keeps its own
replica of the target and serves the requests whose id is congruent to its
rank; rank 0 gathers every result once, in request order, and times the run
as the slowest rank's."""
import os
import socket
import sys
import time

import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    from distributedpanga_b200.serve import Request, Scheduler, serve_sharded
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = [Request(i, b"", 0.01 * i, 1000 * (i + 1)) for i in range(7)]
        seen = []

        def execute(slot, r):
            seen.append(r.rid)
            time.sleep(0.02 * (1 + rank))          # rank 1 is the slow one
            return {"query_bases": r.bases, "gdb_bases": r.bases + 5000}

        def run_local(mine):
            return Scheduler(2, 1 << 40, lambda r: 0).run(mine, execute)

        t = time.monotonic()
        res, summ = serve_sharded(reqs, run_local, rank, world)
        elapsed = time.monotonic() - t
        out[rank] = (sorted(seen), None if res is None else [r.rid for r in res], summ, elapsed)
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_gather():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == [0, 2, 4, 6] and res[1][0] == [1, 3, 5]   # each request served once
    assert res[0][1] == list(range(7))                            # rank 0: all results, in order
    assert res[1][1] is None and res[1][2] is None
    s = res[0][2]
    assert s["requests"] == 7
    assert s["query_mbp_per_s"] > 0 and s["p99_latency_s"] >= s["p50_latency_s"] > 0
    # the run's wall time is the slower rank's: rank 1 sleeps 0.04 s per request
    assert s["wall_s"] >= 0.04 * 2 - 1e-3
    assert abs(s["gdb_mbp_per_s"] * s["wall_s"] - (sum(1000 * (i + 1) for i in range(7)) + 7 * 5000) / 1e6) < 1e-9


def test_one_rank_without_process_group():
    sys.path.insert(0, ROOT)
    from distributedpanga_b200.serve import Request, serve_sharded
    reqs = [Request(i, b"", 0.0, 10) for i in range(3)]
    from distributedpanga_b200.serve import Result
    res, summ = serve_sharded(reqs, lambda mine: [Result(r.rid, 0.0, 0.0, 1.0, 0, {"query_bases": 10})
                                                  for r in reversed(mine)], 0, 1)
    assert [r.rid for r in res] == [0, 1, 2] and summ["requests"] == 3
