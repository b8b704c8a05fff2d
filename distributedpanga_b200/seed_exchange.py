"""Seeds to the rank that owns their contig pair (the reference's stage 3
routing, src/contig_assignment.c, src/seed_exchange.c, src/pga-mpi-merge.c):
after the distributed index build (``dsort.run_stage2``) each rank runs the
adaptamer merge on its own bucket range (``Device.build_kmer_adapter`` and
``Device.self_adaptamer_merge`` on GPUs), then every seed goes to the owner of
(its A contig, its B contig) and each rank holds exactly the seeds of its
pairs, as the single-process merge would have made them.

Seeds are in the reference's byte format: ``[plen][A payload][B payload]``,
each payload ``[position P][contig|strand C]`` little-endian; the A strand
bit is already clear (src/fastga_pipeline.c:365-367, 391-397).

  contig_assignment_build   src/contig_assignment.c:58-133 (pairs i <= j
                            weighted by length product, heaviest first, each
                            to the least loaded rank, ties to the lower rank)
  rank_for_pair             src/pga-mpi-merge.c:446-462 (both (i, j) and
                            (j, i) filled)
  plan_byte_exchange        src/seed_exchange.c:4-24
  redistribute_seeds        the routing of src/fastga_pipeline.c:376-384 and
                            the exchange of src/pga-mpi-merge.c
"""
from __future__ import annotations

import heapq

import numpy as np

INT_MAX = 2 ** 31 - 1


def contig_assignment_build(clen, world_size: int):
    """(owner[i, j] for i <= j (-1 below the diagonal), load per rank)."""
    n = len(clen)
    if world_size <= 0 or n <= 0:
        raise ValueError("contig_assignment_build: no ranks or no contigs")
    if world_size > 127:
        raise ValueError("contig_assignment_build: world size %d > 127" % world_size)
    clen = np.asarray(clen, dtype=np.int64)
    iu, ju = np.triu_indices(n)
    w = clen[iu] * clen[ju]
    order = np.lexsort((ju, iu, -w))                 # weight descending, then (i, j)
    owner = np.full((n, n), -1, dtype=np.int8)
    load = [0] * world_size
    heap = [(0, r) for r in range(world_size)]      # (load, rank): lowest load, then lowest rank
    for k in order:
        ld, r = heap[0]
        owner[iu[k], ju[k]] = r
        load[r] = ld + int(w[k])
        heapq.heapreplace(heap, (load[r], r))
    return owner, np.array(load, dtype=np.int64)


def rank_for_pair(owner: np.ndarray) -> np.ndarray:
    """The symmetric N x N owner table the merge routes by."""
    lo = np.minimum.outer(np.arange(len(owner)), np.arange(len(owner)))
    hi = np.maximum.outer(np.arange(len(owner)), np.arange(len(owner)))
    return owner[lo, hi]


def plan_byte_exchange(sizes):
    """(counts, displs) of a byte exchange, or an error code as the reference
    gives it: -1 a negative size, -2 a size above INT_MAX, -3 a displacement
    above INT_MAX."""
    counts, displs, cum = [], [], 0
    for s in sizes:
        s = int(s)
        if s < 0:
            return -1
        if s > INT_MAX:
            return -2
        if cum + s > INT_MAX:
            return -3
        counts.append(s)
        displs.append(cum)
        cum += s
    return counts, displs


def seed_contigs(seeds: np.ndarray, posb: int, ctgb: int):
    """(A contig, B contig) of each seed, strand bits cleared."""
    def field(off):
        v = np.zeros(len(seeds), dtype=np.int64)
        for b in range(ctgb):
            v |= seeds[:, off + b].astype(np.int64) << (8 * b)
        return v & ((1 << (8 * ctgb - 1)) - 1)
    return field(1 + posb), field(1 + 2 * posb + ctgb)


def redistribute_seeds(seeds: np.ndarray, posb: int, ctgb: int, rfp: np.ndarray, group=None) -> np.ndarray:
    """This rank's seeds of one unit (N or C) after the exchange: the seeds
    every rank made whose pair this rank owns, in source-rank order, each
    source's in its own order."""
    import torch
    import torch.distributed as dist
    from .dsort import _device_of
    world = dist.get_world_size(group)
    dev = _device_of(group)
    sb = 1 + 2 * (posb + ctgb)
    seeds = np.asarray(seeds, dtype=np.uint8).reshape(-1, sb)
    if len(seeds):
        a, b = seed_contigs(seeds, posb, ctgb)
        dest = rfp[a, b].astype(np.int64)
        if dest.min() < 0:
            raise ValueError("a seed's contig pair has no owner")
        order = np.argsort(dest, kind="stable")
        send = seeds[order]
        per = np.bincount(dest, minlength=world) * sb
    else:
        send = seeds
        per = np.zeros(world, dtype=np.int64)
    plan = plan_byte_exchange(per)
    if not isinstance(plan, tuple):
        raise ValueError("plan_byte_exchange: error %d" % plan)
    send_sizes = torch.from_numpy(per.astype(np.int64)).to(dev)
    recv_sizes = torch.zeros(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv_sizes, send_sizes, group=group)
    rs = [int(x) for x in recv_sizes.cpu()]
    out = torch.empty(sum(rs), dtype=torch.uint8, device=dev)
    inp = torch.from_numpy(np.ascontiguousarray(send).reshape(-1)).to(dev)
    dist.all_to_all_single(out, inp, output_split_sizes=rs, input_split_sizes=[int(x) for x in per], group=group)
    return out.cpu().numpy().reshape(-1, sb)
