"""The distributed index build (the reference's stage 2, src/dsort.c) over
torch.distributed: records go to the rank that owns their 10-bit bucket, each
rank sorts what it receives, and the first record of each rank gets its LCP to
the last record of the nearest non-empty rank before it.  Concatenated in rank
order, the ranks' buffers are the single-process sorted index, LCPs included.

Records are in the reference's byte format (``[LCP][k-mer 10][mask][pos
P][contig|strand C]``, src/record.h), as ``Device.extract_to_records`` and
``Device.sort_records`` take and give them.  The exchange runs on the process
group's device: CUDA tensors for NCCL, host tensors for gloo.  The local sort
is a callable: ``Device.sort_records`` (the sm_100a sort) on GPUs, e.g.

    rec = dev.extract_to_records(world, rank)          # this rank's contigs
    mine = run_stage2(rec, lambda r: dev.sort_records(r, posb, ctgb))

Functions keep the reference's names:

  bucket_local_counts            src/dsort.c:108-118
  compute_destination_map        src/dsort.c:120-167 (FastGA's distribute()
                                 splitter with NPARTS = world size)
  organize_send_buffer           src/dsort.c:172-222
  verify_per_rank_sorted         src/dsort.c:227-245
  verify_cross_rank_boundaries   src/dsort.c:247-332
  run_stage2                     src/dsort.c:370-518
"""
from __future__ import annotations

import numpy as np

NUM_BUCK = 1024          # 10-bit buckets: the first five bases
KMER_OFFSET = 1          # the k-mer's bytes follow the LCP byte
KBYTES = 10


class Stage2Error(RuntimeError):
    """A rank's records are out of order, locally or across a rank boundary."""


def record_bucket(kmer_bytes: np.ndarray) -> np.ndarray:
    """The 10-bit bucket of each k-mer: byte 0 and the top two bits of byte 1
    (src/dsort.h:30)."""
    k = kmer_bytes.astype(np.int64)
    return (k[:, 0] << 2) | (k[:, 1] >> 6)


def bucket_local_counts(records: np.ndarray) -> np.ndarray:
    """Records per bucket (int64[NUM_BUCK]); records is (n, record size) uint8."""
    if len(records) == 0:
        return np.zeros(NUM_BUCK, dtype=np.int64)
    return np.bincount(record_bucket(records[:, KMER_OFFSET:KMER_OFFSET + 2]), minlength=NUM_BUCK).astype(np.int64)


def compute_destination_map(global_counts: np.ndarray, world_size: int):
    """(ksplit[world+1], select[NUM_BUCK]): the first bucket of each rank and
    each bucket's rank.  A split falls where the running count crosses
    n * total / world, on whichever side of the crossing bucket is nearer."""
    cum = np.cumsum(np.asarray(global_counts, dtype=np.int64))
    total = int(cum[-1])
    ksplit = [0] * (world_size + 1)
    select = [0] * NUM_BUCK
    n = 1
    t = total // world_size
    for i in range(NUM_BUCK):
        c = int(cum[i])
        if c >= t:
            prev = int(cum[i - 1]) if i > 0 else 0
            if c - t > t - prev:
                select[i] = n
                if n <= world_size:
                    ksplit[n] = i
            else:
                select[i] = n - 1
                if n <= world_size:
                    ksplit[n] = i + 1
            n += 1
            if n > world_size:
                n = world_size
            t = (n * total) // world_size
        else:
            select[i] = n - 1
    ksplit[world_size] = NUM_BUCK
    for r in range(n, world_size):
        ksplit[r] = NUM_BUCK
    return np.array(ksplit, dtype=np.int64), np.array(select, dtype=np.int64)


def organize_send_buffer(records: np.ndarray, select: np.ndarray, world_size: int):
    """Records grouped by destination rank, each group in the local order,
    and the per-rank record counts."""
    if len(records) == 0:
        return records, np.zeros(world_size, dtype=np.int64)
    dest = select[record_bucket(records[:, KMER_OFFSET:KMER_OFFSET + 2])]
    order = np.argsort(dest, kind="stable")
    return records[order], np.bincount(dest, minlength=world_size).astype(np.int64)


def verify_per_rank_sorted(records: np.ndarray):
    """(violations, first bad index or -1): k-mers not in non-decreasing order."""
    if len(records) < 2:
        return 0, -1
    k = records[:, KMER_OFFSET:KMER_OFFSET + KBYTES]
    a, b = k[:-1], k[1:]
    diff = a != b
    first = np.argmax(diff, axis=1)
    has = diff.any(axis=1)
    rows = np.arange(len(a))
    bad = has & (a[rows, first] > b[rows, first])
    idx = np.flatnonzero(bad)
    return int(len(idx)), int(idx[0] + 1) if len(idx) else -1


def kmer_lcp_bases(x: np.ndarray, y: np.ndarray) -> int:
    """Bases two packed 40-mers share from the start (src/sort.c:16-36)."""
    for i in range(KBYTES):
        if x[i] != y[i]:
            d = int(x[i]) ^ int(y[i])
            z = 0
            while not d & (0xc0 >> (2 * z)):
                z += 1
            return 4 * i + z
    return 4 * KBYTES


def _device_of(group=None):
    import torch
    import torch.distributed as dist
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")


def verify_cross_rank_boundaries(records: np.ndarray, group=None, local_bad: int = 0):
    """(boundary violations over all ranks, the last k-mer of the nearest
    non-empty rank before this one or None, local_bad summed over all
    ranks).  Every rank takes the same two collectives whatever its
    records, so a failure anywhere is seen everywhere."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = _device_of(group)
    mine = np.zeros(KBYTES + 1, dtype=np.uint8)
    if len(records):
        mine[0] = 1
        mine[1:] = records[-1, KMER_OFFSET:KMER_OFFSET + KBYTES]
    allv = [torch.zeros(KBYTES + 1, dtype=torch.uint8, device=dev) for _ in range(world)]
    dist.all_gather(allv, torch.from_numpy(mine).to(dev), group=group)
    prev = None
    for r in range(rank - 1, -1, -1):
        v = allv[r].cpu().numpy()
        if v[0]:
            prev = v[1:].copy()
            break
    bad = 0
    if prev is not None and len(records):
        first = records[0, KMER_OFFSET:KMER_OFFSET + KBYTES]
        bad = int(bytes(prev) > bytes(first))
    t = torch.tensor([bad, int(local_bad)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, group=group)
    return int(t[0].item()), prev, int(t[1].item())


def run_stage2(records: np.ndarray, sort_fn, group=None) -> np.ndarray:
    """This rank's slice of the global sorted index from its local records
    ((n, record size) uint8).  `sort_fn(records) -> sorted records with
    LCPs` is the local sort (Device.sort_records on GPUs).  Every rank calls
    it with its own records; collectives in the same order on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = _device_of(group)
    rsize = records.shape[1]
    counts = torch.from_numpy(bucket_local_counts(records)).to(dev)
    dist.all_reduce(counts, group=group)
    _, select = compute_destination_map(counts.cpu().numpy(), world)
    send, per_rank = organize_send_buffer(records, select, world)
    send_sizes = torch.from_numpy(per_rank * rsize).to(dev)
    recv_sizes = torch.zeros(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv_sizes, send_sizes, group=group)
    rs = [int(x) for x in recv_sizes.cpu()]
    ss = [int(x) for x in send_sizes.cpu()]
    out = torch.empty(sum(rs), dtype=torch.uint8, device=dev)
    inp = torch.from_numpy(np.ascontiguousarray(send).reshape(-1)).to(dev)
    dist.all_to_all_single(out, inp, output_split_sizes=rs, input_split_sizes=ss, group=group)
    recv = out.cpu().numpy().reshape(-1, rsize)
    recv = sort_fn(recv) if len(recv) else recv.copy()
    nbad, first_bad = verify_per_rank_sorted(recv)
    boundary_bad, prev, all_bad = verify_cross_rank_boundaries(recv, group, nbad)
    if all_bad:
        raise Stage2Error("local sort check failed: %d violations over all ranks (rank %d: %d, first at %d)"
                          % (all_bad, rank, nbad, first_bad))
    if boundary_bad:
        raise Stage2Error("cross-rank boundary check failed (%d ranks)" % boundary_bad)
    if prev is not None and len(recv):
        recv = recv.copy()
        recv[0, 0] = kmer_lcp_bases(prev, recv[0, KMER_OFFSET:KMER_OFFSET + KBYTES])
    return recv
