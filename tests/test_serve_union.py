"""The rule k_union_rank builds a served request's index by, checked on the
oracle: the sorted index of GDB(target + query) is the merge, by the full
record key (k-mer, then the payload read as one little-endian integer:
contig|strand, then position), of the target's own sorted index -- its
payload widened to the combined GDB's position and contig widths, the strand
bit moved to the top of the wider contig field -- and the query's sorted
records; the LCP bytes are recomputed along the merged order."""
import numpy as np
import pytest

from conftest import load_case


def _le(cols: np.ndarray) -> np.ndarray:
    v = np.zeros(len(cols), dtype=np.int64)
    for b in range(cols.shape[1]):
        v |= cols[:, b].astype(np.int64) << (8 * b)
    return v


def _put_le(out: np.ndarray, off: int, width: int, v: np.ndarray):
    for b in range(width):
        out[:, off + b] = (v >> (8 * b)) & 0xff


def _fields(rec, posb, ctgb):
    pos = _le(rec[:, 12:12 + posb])
    cs = _le(rec[:, 12 + posb:12 + posb + ctgb])
    sign = 1 << (8 * ctgb - 1)
    return pos, cs & (sign - 1), (cs & sign) != 0


def _reencode(rec, posb0, ctgb0, posb1, ctgb1):
    pos, ctg, strand = _fields(rec, posb0, ctgb0)
    out = np.zeros((len(rec), 12 + posb1 + ctgb1), dtype=np.uint8)
    out[:, :12] = rec[:, :12]
    _put_le(out, 12, posb1, pos)
    _put_le(out, 12 + posb1, ctgb1, ctg | (strand.astype(np.int64) << (8 * ctgb1 - 1)))
    return out


def _merge_by_key(rec, posb, ctgb):
    pos = _le(rec[:, 12:12 + posb])
    cs = _le(rec[:, 12 + posb:12 + posb + ctgb])
    keys = [pos, cs] + [rec[:, 10 - j] for j in range(10)]    # last key (k-mer byte 0) is primary
    out = rec[np.lexsort(keys)].copy()
    k = out[:, 1:11]
    lcp = np.zeros(len(out), dtype=np.uint8)
    for i in range(1, len(out)):
        d = np.flatnonzero(k[i] != k[i - 1])
        if len(d) == 0:
            lcp[i] = 40
        else:
            x, z = int(k[i, d[0]] ^ k[i - 1, d[0]]), 0
            while not x & (0xc0 >> (2 * z)):
                z += 1
            lcp[i] = 4 * d[0] + z
    out[:, 0] = lcp
    return out


@pytest.mark.parametrize("case,nt", [("small_s002", 7), ("edge_mix", 9), ("many_contigs", 100)])
def test_union_of_sorted_indices_is_the_combined_index(oracle, case, nt):
    from distributedpanga_b200 import gdb
    cs, _ = load_case(case)
    contigs = [cs.contig(i) for i in range(cs.ncontig)]
    T, U = gdb.from_contigs(contigs[:nt]), gdb.from_contigs(contigs)
    tp, tc, _ = gdb.record_sizing(T)
    up, uc, _ = gdb.record_sizing(U)
    t_idx = oracle.sort_records(oracle.extract(T, tp, tc))
    u_all = oracle.extract(U, up, uc)
    q = u_all[_fields(u_all, up, uc)[1] >= nt]
    merged = _merge_by_key(np.concatenate([_reencode(t_idx, tp, tc, up, uc), oracle.sort_records(q)]), up, uc)
    want = oracle.sort_records(u_all)
    assert np.array_equal(merged, want)
    if case == "many_contigs":
        assert (tc, uc) == (1, 2)                          # the contig field widens in the union
