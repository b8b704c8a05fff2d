"""The distributed index build's device path: one rank over NCCL (CUDA
tensors for the exchange), the sm_100a sort as the local sort, records from
the device extraction; equal to the oracle's sorted index."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_stage2_one_rank_over_nccl(dev, oracle):
    import torch
    import torch.distributed as dist
    from conftest import load_case
    from distributedpanga_b200 import dsort, gdb
    cs, _ = load_case("edge_mix")
    posb, ctgb, _ = gdb.record_sizing(cs)
    dev.gdb_load(cs)
    rec = dev.extract_to_records(1, 0)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0, world_size=1)
    try:
        got = dsort.run_stage2(rec, lambda r: dev.sort_records(r, posb, ctgb))
    finally:
        dist.destroy_process_group()
    want = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    assert np.array_equal(got, want)
