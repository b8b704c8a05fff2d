"""The restated aligner (align_core.cuh, the code the GPU kernel's chain
driver shares) run on the host from the oracle's diagonal-sorted seeds: its
alignments must be the reference's .1aln record stream, record for record.
Self pairs start from the entry values of FastGA's order rules
(src/fastga_order_core.c), computed here in Python from the host results."""
import ctypes as C
import gzip
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, ROOT, load_case

NATIVE = os.path.join(ROOT, "tests", "native")
ALL_CASES = GOLDEN_CASES + ["small_full"]


def load_aht():
    """The host aligner harness (tests/native/align_host.cu), rebuilt when a
    source is newer than the library."""
    so = os.path.join(NATIVE, "libalign_host.so")
    src = os.path.join(NATIVE, "align_host.cu")
    deps = [src, os.path.join(ROOT, "oracle", "scalar_align.cuh")] + [
        os.path.join(ROOT, "distributedpanga_b200", "csrc", f) for f in ("align_core.cuh", "align_spec.h", "finish.cuh")]
    if not os.path.exists(so) or any(os.path.getmtime(d) > os.path.getmtime(so) for d in deps):
        subprocess.run(["/usr/local/cuda/bin/nvcc", "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                        "-Wno-deprecated-gpu-targets", "-o", so, src], check=True)
    L = C.CDLL(so)
    vp, i64, ci = C.c_void_p, C.c_int64, C.c_int
    L.aht_align_unit.argtypes = [vp, ci, vp, vp, vp, vp, vp, ci, ci, ci, ci, vp, ci, i64, i64, vp, i64, vp, vp,
                                 i64, vp, vp, i64, vp, i64]
    L.aht_align_unit.restype = ci
    L.aht_set_finish.argtypes = [ci]
    L.aht_set_finish.restype = None
    L.aht_finish_check.argtypes = [i64, vp, vp, vp, i64, ci, vp, vp, vp, vp]
    L.aht_finish_check.restype = ci
    return L


@pytest.fixture(scope="module")
def aht():
    return load_aht()


def run_unit(L, cs, arr, off, dig, comp, self_entry=None, split=0):
    rows = np.zeros((400000, 9), np.int32)
    tr = np.zeros(64_000_000, np.uint8)
    pairs = np.zeros((200000, 4), np.int32)
    nr, nt, npair = C.c_int64(), C.c_int64(), C.c_int64()
    se = None if self_entry is None else np.ascontiguousarray(self_entry, np.int32)
    rc = L.aht_align_unit(cs.bps.ctypes.data, cs.ncontig, cs.clen.ctypes.data, cs.boff.ctypes.data,
                          cs.freq.ctypes.data, np.ascontiguousarray(arr).ctypes.data, off.ctypes.data,
                          dig["swide"], dig["dbyte"], dig["ctgb"], comp,
                          se.ctypes.data if se is not None else None, 8192, 50_000_000, 1_000_000,
                          rows.ctypes.data, len(rows), C.byref(nr), tr.ctypes.data, len(tr), C.byref(nt),
                          pairs.ctypes.data, len(pairs), C.byref(npair), split)
    assert rc == 0, rc
    out, o = [], 0
    for r in rows[: nr.value]:
        t = tr[o:o + r[8]]
        o += r[8]
        out.append((int(r[0]), int(r[3]), int(r[1]), int(r[2]), int(r[4]), int(r[5]), int(r[6]), int(r[7]),
                    t[1::2].tolist(), t[0::2].tolist()))
    return out, pairs[: npair.value].copy()


def fastga_self_entries(cs, pairs_n, nseeds_by_contig, swide, perm):
    """Entry bepos of every self pair (src/fastga_order_core.c:147-192)."""
    n = cs.ncontig
    pos = np.empty(n, int)
    pos[perm] = np.arange(n)
    clen_pos = cs.clen[perm]
    seeds_pos = nseeds_by_contig[perm]
    T, npost = 32, int(cs.clen.sum())
    split, p, r, t, cum = [0] * (T + 1), 0, T, npost // T, int(clen_pos[0]) if n else 0
    for x in range(1, n):
        if cum >= t and x >= r:
            p += 1
            split[p] = x
            t = (npost * (p + 1)) // T
            r += T
        cum += int(clen_pos[x])
    nparts = p + 1
    split[nparts] = n
    rs = list(range(n))
    for i in range(nparts):
        asize = sum(int(seeds_pos[x]) * swide for x in range(split[i], split[i + 1]))
        if asize == 0:
            continue
        k, thr, s = 0, asize // T, 0
        x = split[i]
        while x < split[i + 1] and seeds_pos[x] == 0:
            x += 1
        beg = x
        while x < split[i + 1]:
            if seeds_pos[x] > 0:
                s += int(seeds_pos[x]) * swide
                if s >= thr:
                    for y in range(beg, x + 1):
                        rs[y] = beg
                    k += 1
                    thr = (asize * (k + 1)) // T
                    beg = x + 1
            x += 1
    res = {(int(a), int(b)): (int(c), int(e)) for a, b, c, e in pairs_n}
    Lk = [0] * n
    for (a, b), (calls, bep) in res.items():
        if a != b and calls > 0:
            key = ((int(pos[b]) + 1) << 32) | (bep & 0xffffffff)
            Lk[pos[a]] = max(Lk[pos[a]], key)
    return pos, rs, res, Lk


def aln_lines(out):
    out = sorted(out, key=lambda x: (x[0], x[1], x[2], x[3]))
    return ["%d %d %d %d %d %d %d %d ; %s ; %s" % (a, ab, ae, b, bb, be, c, d, " ".join(map(str, T)),
                                                   " ".join(map(str, X)))
            for (a, ab, b, c, ae, bb, be, d, T, X) in out]


@pytest.mark.parametrize("case", ALL_CASES)
def test_host_aligner_matches_reference(oracle, aht, case):
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    srt = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    ent, cum, _ = oracle.build_adapter(srt, posb, ctgb)
    ns, css, nb, _ = oracle.merge(ent, cum, posb, ctgb, 10, cs.ncontig)
    arrN, offN = oracle.reimport_sort(ns, posb, ctgb, 0, cs.ncontig, cs.maxctg, dig["dbyte"])
    arrC, offC = oracle.reimport_sort(css, posb, ctgb, 1, cs.ncontig, cs.maxctg, dig["dbyte"])
    # pass 1: every pair; the results of pairs of two contigs fix the self pairs' entry values
    perm = np.argsort(-cs.clen, kind="stable")
    assert perm.tolist() == dig["gix_perm"]           # FastGA's contig order = the .gix permutation
    _, pairsN = run_unit(aht, cs, arrN, offN, dig, 0)
    pos, rs, res, Lk = fastga_self_entries(cs, pairsN, nb, dig["swide"], perm)
    entry = np.zeros(cs.ncontig, np.int32)
    S = [0] * cs.ncontig
    selfs = sorted([a for (a, b) in res if a == b], key=lambda c: pos[c])
    known = {}
    for c in selfs:
        x = pos[c]
        S[x] = 1
        earlier = sorted([(pos[b], res[(c, b)]) for (a, b) in res if a == c and pos[b] < x], reverse=True)
        v = next((bep for _, (calls, bep) in earlier if calls > 0), None)
        if v is not None:
            known[c] = v
        elif rs[x] == x:
            known[c] = 32767 if rs[x] == 0 else 0
    # self pairs whose value comes from earlier rows: resolve in rounds
    for c in selfs:
        if c in known:
            entry[c] = known[c]
    for _ in range(len(selfs) + 1):
        _, pairsN = run_unit(aht, cs, arrN, offN, dig, 0, entry)
        res = {(int(a), int(b)): (int(cc), int(e)) for a, b, cc, e in pairsN}
        for c in selfs:
            if c in known:
                calls, bep = res[(c, c)]
                S[pos[c]] = 3 + bep if calls > 0 else 2
        progress = False
        for c in selfs:
            if c in known:
                continue
            x = pos[c]
            val, wait = None, False
            for y in range(x - 1, rs[x] - 1, -1):
                k, s = Lk[y], S[y]
                if k and (k >> 32) - 1 > y:
                    val = k & 0xffffffff
                elif s == 1:
                    wait = True
                elif s >= 3:
                    val = s - 3
                elif k:
                    val = k & 0xffffffff
                else:
                    continue
                break
            if wait:
                continue
            known[c] = val if val is not None else (32767 if rs[x] == 0 else 0)
            entry[c] = known[c]
            progress = True
        if not progress:
            break
    outN, _ = run_unit(aht, cs, arrN, offN, dig, 0, entry)
    outC, _ = run_unit(aht, cs, arrC, offC, dig, 1)
    mine = [" ".join(l.split()) for l in aln_lines(outN + outC)]
    ref = [" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n")
           if l.strip()]
    assert len(mine) == dig["aln"]["count"]
    assert mine == ref


@pytest.mark.parametrize("case", ["small_s002", "chromset_s0005", "edge_mix", "small_full"])
def test_host_block_ranges_compose(oracle, aht, case):
    """Splitting each pair of two different contigs into consecutive band
    ranges (as the GPU does with large pairs) and concatenating the ranges'
    candidates gives the whole-pair run's output, record for record and in
    the same order, and the same calls and exit bepos per pair."""
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    srt = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    ent, cum, _ = oracle.build_adapter(srt, posb, ctgb)
    ns, css, _, _ = oracle.merge(ent, cum, posb, ctgb, 10, cs.ncontig)
    for comp, seeds in ((0, ns), (1, css)):
        arr, off = oracle.reimport_sort(seeds, posb, ctgb, comp, cs.ncontig, cs.maxctg, dig["dbyte"])
        whole, pw = run_unit(aht, cs, arr, off, dig, comp)
        for split in (1, 13, 200):
            part, pp = run_unit(aht, cs, arr, off, dig, comp, split=split)
            assert len(part) == len(whole)
            assert part == whole, (comp, split)
            assert np.array_equal(pp, pw), (comp, split)


# ---- the finishing step against the oracle's statement-by-statement restatement

def _random_candidates(rng, n, base_len=30000, T=100):
    """n candidate alignments of one pair, drawn around one base path so that
    they share starts and ends (duplicates, containments), meet at trace
    points (crossings) and run beside each other at small B offsets (boxes).
    Returns rows6 (abpos aepos bbpos bepos diffs tlen), trace offsets and the
    trace bytes ((diffs, b-delta) per A panel)."""
    npan = base_len // T + 1
    bd = 100 + rng.integers(-4, 5, npan)
    at = np.concatenate([[0], np.cumsum(bd)])

    def bpos(x):
        return int(at[x // T] + (bd[x // T] * (x % T)) // T)

    rows, offs, tr = [], [], []
    nb = 0
    for i in range(n):
        u = rng.random()
        if rows and u < 0.12:                       # an exact copy of an earlier one
            k = int(rng.integers(0, len(rows)))
            r = list(rows[k])
            t = tr[k].copy()
            if rng.random() < 0.5:                  # ... with other diffs
                t[0::2] = rng.integers(0, 12, len(t) // 2)
                r[4] = int(t[0::2].sum())
            rows.append(r)
            tr.append(t)
            offs.append(nb)
            nb += len(t)
            continue
        if rows and u < 0.3:                        # same start or same end as an earlier one
            k = int(rng.integers(0, len(rows)))
            a0, a1 = rows[k][0], rows[k][1]
            if rng.random() < 0.5:
                a1 = int(min(base_len, a0 + rng.integers(150, 8000)))
            else:
                a0 = int(max(0, a1 - rng.integers(150, 8000)))
            off = rows[k][2] - bpos(rows[k][0])
        else:
            a0 = int(rng.integers(0, base_len - 400))
            a1 = int(min(base_len, a0 + rng.integers(150, 9000)))
            off = int(rng.choice([0, 0, 0, 1, -2, 3, 12, -15]))
        p0, p1 = a0 // T, (a1 - 1) // T
        deltas = []
        for p in range(p0, p1 + 1):
            s, e = max(a0, p * T), min(a1, (p + 1) * T)
            deltas.append(bpos(e) - bpos(s))
        deltas = np.array(deltas, np.int64)
        if len(deltas) > 2 and rng.random() < 0.4:  # wander off the path and come back
            q = int(rng.integers(0, len(deltas) - 1))
            w = int(rng.integers(q + 1, len(deltas)))
            h = int(rng.integers(1, 4)) * (1 if rng.random() < 0.5 else -1)
            deltas[q] += h
            deltas[w] -= h
        deltas = np.clip(deltas, 0, 255)
        diffs = rng.integers(0, 12, len(deltas))
        t = np.zeros(2 * len(deltas), np.uint8)
        t[0::2] = diffs
        t[1::2] = deltas
        b0 = bpos(a0) + off
        rows.append([a0, a1, b0, b0 + int(deltas.sum()), int(diffs.sum()), len(t)])
        tr.append(t)
        offs.append(nb)
        nb += len(t)
    return (np.array(rows, np.int32).reshape(-1, 6), np.array(offs, np.int64),
            np.concatenate(tr) if tr else np.zeros(1, np.uint8))


def _finish(L, rows, offs, tr, which):
    n = len(rows)
    out = np.zeros((max(1, n), 6), np.int32)
    otr = np.zeros(max(1, 4 * tr.size), np.uint8)
    on, ob = C.c_int64(), C.c_int64()
    rc = L.aht_finish_check(n, np.ascontiguousarray(rows).ctypes.data, offs.ctypes.data, tr.ctypes.data, tr.size,
                            which, out.ctypes.data, C.byref(on), otr.ctypes.data, C.byref(ob))
    assert rc == 0
    return out[: on.value].copy(), otr[: ob.value].copy()


@pytest.mark.parametrize("seed", range(12))
def test_finishing_step_matches_oracle_rules(aht, seed):
    """The product's finishing step (finish.cuh, lanes emulated on the host)
    against the oracle's statement-by-statement restatement of the
    reference's sort / elimination / entwine / box rules, on random candidate
    sets built to hit every rule (sizes 1 to 400, crossing the 32-lane
    windows)."""
    rng = np.random.default_rng(1000 + seed)
    hits = 0
    for n in (1, 2, 5, 31, 33, 64, 150, 400):
        rows, offs, tr = _random_candidates(rng, n)
        got = _finish(aht, rows, offs, tr, 0)
        want = _finish(aht, rows, offs, tr, 1)
        assert np.array_equal(got[0], want[0]), (seed, n)
        assert np.array_equal(got[1], want[1]), (seed, n)
        hits += n - len(want[0])
    assert hits > 0   # some candidates were removed or joined
