"""FastGA's order of self pairs across ranks: the sharded path's last exchange.

Reference: the rules of src/fastga_order_core.c:50-192 (fo_compute_ranges,
the entry value of a self pair from the nearest earlier partner that called,
fo_from_rows) and the protocol of src/fastga_order.c:1-45,185-262: there
every pair (x, b) with b earlier in the order sends its outcome to the self
pair's owner in a point-to-point message, so that a self pair can start as
soon as its nearest calling partner has answered, and the rest is resolved
in rounds of two MPI_MAX all-reduces (L and S below).  Here the answers are
one more all-reduce (eb), taken once every pair of two contigs has run: the
values are the same, the self pairs start later (they are about 1/ncontig of
a unit's pairs), and there are no messages to poll for.

Each rank aligns the contig pairs it owns (seed_exchange's assignment).  A
self pair (c, c) of the N unit starts from an entry bepos that depends on
the calls of other pairs, which other ranks may own.  Every per-contig value
the rules read is a maximum over pairs, so here they are combined across
ranks with one all-reduce(MAX) each -- a rank that owns none of the pairs
contributes 0 -- indexed by the contig's position x in FastGA's order:

  lk[x]  the largest order key (pos[b] + 1) << 32 | exit bepos over the N
         pairs (a, b), a != b, a = the contig at x, that made a call;
  eb[x]  the same over the partners earlier in the order (pos[b] < x);
  st[x]  the state of the self pair at x: 0 none, 1 pending, 2 aligned with
         no call, 3 + exit bepos aligned with a call (a state only grows).

A self pair whose value the rules can only take from an earlier self pair's
outcome is resolved in rounds: every rank decides the same entry values
from the combined arrays, the owners align those self pairs, and the new
states are all-reduced before the next round.
"""
from __future__ import annotations

import numpy as np

UNSET_MAIN = 32767  # the entry value of a self pair at the start of the first range


def order_positions(clen):
    """FastGA's contig order (GIXmake's: longest first, ties by number) as
    (perm, pos): perm[x] is the contig at position x, pos[c] its position."""
    clen = np.asarray(clen, dtype=np.int64)
    perm = np.argsort(-clen, kind="stable")
    pos = np.empty(len(clen), dtype=np.int64)
    pos[perm] = np.arange(len(clen))
    return perm, pos


def range_starts(clen, seeds_by_contig, swide: int, perm, nthreads: int = 32) -> list:
    """rs[x]: the first position of the order range that position x falls in
    (fo_compute_ranges, src/fastga_order_core.c:50-140): the order is cut
    into parts of about equal sequence, each part into ranges of about equal
    seed bytes.  The library's own rule, the one pga_align uses
    (pga_fastga_ranges)."""
    import ctypes as C
    from . import pipeline
    n = len(clen)
    if n == 0:
        return []
    clen = np.asarray(clen, dtype=np.int64)
    cp = np.ascontiguousarray(clen[perm])
    sp = np.ascontiguousarray(np.asarray(seeds_by_contig, dtype=np.int64)[perm])
    rs = np.zeros(n, dtype=np.int32)
    rc = pipeline.load_library().pga_fastga_ranges(n, cp.ctypes.data_as(C.c_void_p), int(clen.sum()),
                                                   sp.ctypes.data_as(C.c_void_p), int(swide), int(nthreads),
                                                   rs.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise pipeline.PgaError("pga_fastga_ranges: status %d" % rc)
    return rs.tolist()


def local_keys(pairs_n, pos, n: int):
    """(lk, eb) from this rank's N-pair outcomes: rows (a, b, calls, exit
    bepos) of the pairs it aligned."""
    lk = np.zeros(n, dtype=np.int64)
    eb = np.zeros(n, dtype=np.int64)
    for a, b, calls, bep in pairs_n:
        a, b = int(a), int(b)
        if a == b or calls <= 0:
            continue
        xa, xb = int(pos[a]), int(pos[b])
        key = ((xb + 1) << 32) | (int(bep) & 0xffffffff)
        lk[xa] = max(lk[xa], key)
        if xb < xa:
            eb[xa] = max(eb[xa], key)
    return lk, eb


def first_values(st, eb, rs) -> dict:
    """Entry values known before any self pair is aligned, by position: the
    nearest earlier partner that called (src/fastga_order_core.c:147-166),
    or, at the start of a range, the unset value."""
    known = {}
    for x in range(len(st)):
        if st[x] != 1:
            continue
        if eb[x] != 0:
            known[x] = int(eb[x] & 0xffffffff)
        elif rs[x] == x:
            known[x] = UNSET_MAIN if rs[x] == 0 else 0
    return known


def from_rows(x: int, lk, st, rs):
    """fo_from_rows (src/fastga_order_core.c:167-192) for the self pair at
    x: (value, wait).  wait: an earlier self pair in x's range is still
    pending; value None: nothing earlier decides it (the unset value)."""
    for y in range(x - 1, rs[x] - 1, -1):
        k, s = int(lk[y]), int(st[y])
        if k and (k >> 32) - 1 > y:
            return k & 0xffffffff, False
        if s == 1:
            return None, True
        if s >= 3:
            return s - 3, False
        if k:
            return k & 0xffffffff, False
    return None, False


def resolve(n: int, pos, rs, lk, eb, st, align_round, allreduce_max):
    """(entry values of every self pair by contig, rounds).

    lk, eb, st: the all-reduced arrays after the pairs of two contigs were
    aligned (st holds 1 at every self pair, 0 elsewhere).  align_round(entry)
    aligns, on this rank, the self pairs it owns among those whose entry is
    given (entry: contig -> value, the ones decided since the last round) and
    returns their outcomes {contig: (calls, exit bepos)}; allreduce_max(array)
    combines an int64 array across ranks.  Every rank calls this with the
    same arrays, decides the same values and takes the same collective steps.

    The earliest undecided self pair of a range always has a value (nothing
    before it in the range is pending), so every round decides at least one
    until none is left.  A self pair decided but reported by no rank stays
    pending and raises, on every rank alike."""
    pos = np.asarray(pos)
    perm = np.empty(n, dtype=np.int64)
    perm[pos] = np.arange(n)
    st = np.array(st, dtype=np.int64)

    def decide(known):
        new = {}
        for x in range(n):
            if st[x] != 1 or x in known:
                continue
            val, wait = from_rows(x, lk, st, rs)
            if not wait:
                new[x] = val if val is not None else (UNSET_MAIN if rs[x] == 0 else 0)
        return new

    known = first_values(st, eb, rs)
    known.update(decide(known))
    new, rounds = dict(known), 0
    while new:
        rounds += 1
        out = align_round({int(perm[x]): v for x, v in new.items()})
        mine = np.zeros(n, dtype=np.int64)
        for c, (calls, bep) in out.items():
            mine[pos[c]] = 3 + int(bep) if calls > 0 else 2
        st = np.maximum(st, allreduce_max(mine))
        new = decide(known)
        known.update(new)
    if (st == 1).any():
        raise RuntimeError("self pairs at order positions %s were left pending" % np.nonzero(st == 1)[0][:8].tolist())
    return {int(perm[x]): v for x, v in known.items()}, rounds
