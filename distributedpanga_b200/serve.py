"""The served form: a request loop over one resident target.

A target assembly is ingested and indexed once (``pipeline.Target``) and
stays in HBM.  A request is a query assembly (FASTA text); its result is the
plain path's on the GDB that the target's text followed by the query's makes
(``Device.serve_load`` builds that GDB and its index by merging the query's
sorted k-mer records into the target's, then the request runs the adaptamer
merge, the diagonal sort and the alignment as any GDB does).  Every pair of
that GDB is aligned: the frequency cutoff counts k-mers over both
assemblies and FastGA's self-pair order looks across all contigs, so a
request's alignments cannot be restricted to pairs with a query contig and
stay equal to the plain run's.

Scheduling is continuous batching.  Requests arrive on their own clock (a
Poisson stream in the benchmark).  The dispatcher admits the oldest waiting
request as soon as a slot is free and the device memory it needs fits the
budget.  A slot is one context (its own CUDA stream) driven by its own host
thread.  Admitted requests run at the same time: their kernels share the
device through their streams, so one request's sort, merge or alignment
kernels take the SMs that another's leave idle (the alignment launches end
in a tail of long pairs).  Contexts keep their buffers between requests and
only grow them, so a slot holds the largest footprint it has served: the
budget is charged that high-water mark per slot, not only what is in flight.
A request whose footprint alone exceeds the budget still runs when nothing
else is in flight.  Requests never overtake each other at admission (FIFO),
so a large request is not starved by small ones behind it.

Each result is the same alone and in the mix: a request owns its context
for its whole run and the target is never written after it is built.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np

# Device bytes a request holds per base of GDB(target + query): k-mer records
# and their sorted copy (2 x 16 B x ~0.8 records/base), LCPs and seeds, the
# diagonal-sort keys, and the aligner's sequences and pools; plus a fixed part
# (the 2^24-entry prefix tables and scratch).
BYTES_PER_BASE = 64
FIXED_BYTES = 1 << 30


def footprint_bytes(gdb_bases: int, bytes_per_base: float = BYTES_PER_BASE) -> int:
    return int(bytes_per_base * int(gdb_bases)) + FIXED_BYTES


@dataclass
class Request:
    rid: int
    text: bytes          # the query assembly's FASTA text
    arrival: float       # seconds after the stream starts
    bases: int           # the query's bases


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    done: float
    slot: int
    out: dict = field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class Scheduler:
    """FIFO admission of timed requests into `slots` concurrent slots under a
    device-memory budget.  `execute(slot, request) -> dict` runs one request
    on a slot's context; it is called on that slot's own thread."""

    def __init__(self, slots: int, budget_bytes: int, footprint):
        if slots < 1:
            raise ValueError("at least one slot")
        self.slots = slots
        self.budget = int(budget_bytes)
        self.footprint = footprint
        self.held = [0] * slots          # high-water footprint per slot

    def charge_if_admitted(self, slot: int, need: int) -> int:
        """Budget in use if `slot` takes a request needing `need` bytes."""
        return sum(self.held) - self.held[slot] + max(self.held[slot], need)

    def pick_slot(self, free: list, need: int, in_flight: int):
        """The free slot to admit into, or None: a slot that already holds
        `need` first (no growth), else the one whose growth fits the budget
        best; anything goes when nothing is in flight."""
        ok = [s for s in free if self.charge_if_admitted(s, need) <= self.budget]
        if not ok:
            if in_flight == 0 and free:
                ok = free
            else:
                return None
        fits = [s for s in ok if self.held[s] >= need]
        if fits:
            return min(fits, key=lambda s: self.held[s])
        return min(ok, key=lambda s: self.charge_if_admitted(s, need))

    def run(self, requests: list, execute, clock=time.monotonic, wait=None) -> list:
        """Runs `requests` (arrival-ordered) as they arrive; returns their
        Results in request order.  A failure in any request is raised after
        the requests in flight have finished."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        cv = threading.Condition()
        free = list(range(self.slots))
        results, errors, threads = {}, [], []
        t0 = clock()
        state = {"in_flight": 0}

        def worker(slot, req, admitted):
            try:
                out = execute(slot, req)
                err = None
            except BaseException as e:  # raised on the caller's thread below
                out, err = None, e
            with cv:
                done = clock() - t0
                if err is None:
                    results[req.rid] = Result(req.rid, req.arrival, admitted, done, slot, out)
                else:
                    errors.append(err)
                free.append(slot)
                state["in_flight"] -= 1
                cv.notify_all()

        i = 0
        with cv:
            while i < len(reqs) or state["in_flight"] > 0:
                now = clock() - t0
                while i < len(reqs) and not errors and reqs[i].arrival <= now:
                    need = self.footprint(reqs[i])
                    slot = self.pick_slot(free, need, state["in_flight"])
                    if slot is None:
                        break
                    free.remove(slot)
                    self.held[slot] = max(self.held[slot], need)
                    state["in_flight"] += 1
                    th = threading.Thread(target=worker, args=(slot, reqs[i], now), daemon=True)
                    threads.append(th)
                    th.start()
                    i += 1
                if errors and state["in_flight"] == 0:
                    break
                if i < len(reqs) and not errors and free and reqs[i].arrival > now:
                    timeout = reqs[i].arrival - now
                else:
                    timeout = None if state["in_flight"] > 0 else 0.0
                if wait is not None:
                    wait(cv, timeout)
                else:
                    cv.wait(timeout)
        for th in threads:
            th.join()
        if errors:
            raise errors[0]
        return [results[r.rid] for r in requests]


def summarize(results: list, wall_s: float) -> dict:
    """Throughput and per-request latency of a served run."""
    lat = np.array([r.latency for r in results], dtype=np.float64)
    qb = sum(int(r.out.get("query_bases", 0)) for r in results)
    gb = sum(int(r.out.get("gdb_bases", 0)) for r in results)
    return {
        "requests": len(results),
        "wall_s": wall_s,
        "query_mbp_per_s": qb / 1e6 / wall_s if wall_s > 0 else 0.0,
        "gdb_mbp_per_s": gb / 1e6 / wall_s if wall_s > 0 else 0.0,
        "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else 0.0,
        "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else 0.0,
        "mean_latency_s": float(lat.mean()) if len(lat) else 0.0,
    }


class Server:
    """The request loop on one device: `slots` contexts serving requests
    against `target` (a pipeline.Target), FIFO under `budget_bytes` of device
    memory (default: what the device has free when the server starts, less
    the target-independent reserve of 4 GiB), a request charged
    `bytes_per_base` per base of GDB(target + query) (a measured figure where
    the caller has one: see bench.py's served measurement)."""

    def __init__(self, target, slots: int = 2, budget_bytes: int | None = None, freq: int = 10,
                 keep_alignments: bool = True, bytes_per_base: float = BYTES_PER_BASE):
        from . import pipeline
        self.target = target
        self.freq = freq
        self.keep = keep_alignments
        self.devs = [pipeline.Device(target.device) for _ in range(slots)]
        if budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info(target.device)
            budget_bytes = max(0, free - (4 << 30))
        tb = target.bases
        self.sched = Scheduler(slots, budget_bytes, lambda r: footprint_bytes(tb + r.bases, bytes_per_base))

    def close(self):
        for d in self.devs:
            d.close()
        self.devs = []

    def execute(self, slot: int, req: Request) -> dict:
        d = self.devs[slot]
        sizes = d.serve_load(self.target, req.text)
        d.merge(self.freq)
        n = d.align()
        out = {"nalign": n, "gdb_bases": int(sizes[5]), "query_bases": int(sizes[5]) - self.target.bases,
               "records": d.nrec, "reuse": d.reuse_stats()}
        if self.keep:
            out["alignments"] = d.alignments()
        return out

    def run(self, requests: list) -> tuple:
        t = time.monotonic()
        res = self.sched.run(requests, self.execute)
        wall = time.monotonic() - t
        return res, summarize(res, wall)


def plain_request(dev, target_text: bytes, query_text: bytes, nthr: int = 0, freq: int = 10) -> dict:
    """The plain path for one request on `dev`: ingest of the target's text
    followed by the query's, index build, merge and alignment (what a request
    costs without a resident target)."""
    dev.gdb_ingest_fasta(target_text + query_text, nthr=nthr, tables=False)
    dev.index_build(want_entries=False)
    dev.merge(freq)
    n = dev.align()
    return {"nalign": n, "alignments": dev.alignments(), "records": dev.nrec}


def shard(requests: list, rank: int, world: int) -> list:
    """The requests rank `rank` of `world` serves: request ids congruent to
    the rank (each GPU keeps its own replica of the target)."""
    return [r for r in requests if r.rid % world == rank]


def serve_sharded(requests: list, run_local, rank: int, world: int) -> tuple:
    """Runs this rank's share of `requests` with `run_local(reqs) -> results`
    between two barriers and gathers every rank's results on rank 0, which
    gets (all results in request order, summary with wall = the slowest
    rank's); other ranks get (None, None).  Without an initialised process
    group (world 1) it is run_local and summarize."""
    import torch.distributed as dist
    mine = shard(requests, rank, world)
    dist_on = world > 1 and dist.is_available() and dist.is_initialized()
    if dist_on:
        dist.barrier()
    t = time.monotonic()
    res = run_local(mine)
    wall = time.monotonic() - t
    if dist_on:
        dist.barrier()
        box = [None] * world
        dist.all_gather_object(box, (wall, res))
        if rank != 0:
            return None, None
        wall = max(w for w, _ in box)
        res = [r for _, rs in box for r in rs]
    order = {r.rid: i for i, r in enumerate(requests)}
    res.sort(key=lambda r: order[r.rid])
    return res, summarize(res, wall)
