"""The bench's multi-rank plumbing on CPU: world size 2 over gloo.  Each rank
runs its own replica; the timed values are combined as the maximum over
ranks, only rank 0 prints, and the reference arm does its work on rank 0
alone."""
import io
import os
import socket
import sys
import contextlib

import pytest
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
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        ms, e2e = bench.max_over_ranks([10.0 + rank, 20.0 - rank], world, "cpu")
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            bench.emit(rank, {"rank": rank, "ms": ms})
        # the reference arm: ranks other than 0 return at once
        args = type("A", (), {"ref_scale": 0.02, "warmup": 3, "steps": 1, "gpus": world})()
        if rank != 0:
            with contextlib.redirect_stdout(io.StringIO()) as ref_out:
                bench.run_reference(args, rank)
            ref_printed = ref_out.getvalue()
        else:
            ref_printed = ""
        bench.barrier(world)
        out[rank] = (ms, e2e, buf.getvalue(), ref_printed)
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_and_single_line():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == 11.0 and res[1][0] == 11.0      # max of 10, 11
    assert res[0][1] == 20.0 and res[1][1] == 20.0      # max of 20, 19
    assert res[0][2].strip().startswith("{") and '"rank": 0' in res[0][2]
    assert res[1][2] == ""                               # rank 1 prints nothing
    assert res[1][3] == ""                               # reference arm: rank 1 idle


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1, "cpu") == [1.5, 2.5]
    bench.barrier(1)
