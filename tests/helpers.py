"""Digest helpers shared by the oracle and GPU parity tests."""
import hashlib

import numpy as np


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix64(z: np.ndarray) -> np.ndarray:
    """splitmix64's finaliser, element-wise on uint64 (wrapping arithmetic)."""
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def multiset_digest(rows: np.ndarray, chunk: int = 1 << 22) -> str:
    """Order-independent digest of the rows of a 2-D uint8 array: each row is
    hashed (its bytes as little-endian 64-bit words, zero-padded, chained
    through splitmix64's finaliser), and the digest is the row count with the
    wrapping sum of the row hashes and the wrapping sum of a second mix of
    them.  Equal multisets give equal digests; for the large cases, where a
    full lexicographic sort of the rows would take minutes."""
    n, w = rows.shape
    nw = (w + 7) // 8
    s1 = np.uint64(0)
    s2 = np.uint64(0)
    with np.errstate(over="ignore"):
        for lo in range(0, n, chunk):
            blk = rows[lo:lo + chunk]
            pad = np.zeros((blk.shape[0], nw * 8), np.uint8)
            pad[:, :w] = blk
            words = pad.view("<u8")
            h = np.full(blk.shape[0], 0x9E3779B97F4A7C15, np.uint64)
            for j in range(nw):
                h = _mix64(h ^ (words[:, j] + np.uint64(j + 1) * _M2))
            s1 = s1 + h.sum(dtype=np.uint64)
            s2 = s2 + _mix64(h ^ _M1).sum(dtype=np.uint64)
    return "%d:%016x:%016x" % (n, int(s1), int(s2))


def lines_digest(lines, block: int = 1000) -> dict:
    """sha256 of a record stream (lines joined by newlines), with one sha per
    block of `block` lines so that a mismatch can be located."""
    blocks = [hashlib.sha256("\n".join(lines[i:i + block]).encode()).hexdigest()[:16]
              for i in range(0, len(lines), block)]
    return {"count": len(lines), "sha": hashlib.sha256("\n".join(lines).encode()).hexdigest(), "block": block,
            "block_sha": blocks}


def canonical_rows(a: np.ndarray) -> np.ndarray:
    if a.shape[0] == 0:
        return a
    v = np.ascontiguousarray(a).view(np.dtype((np.void, a.shape[1]))).reshape(-1)
    return a[np.argsort(v, kind="stable")]


def prefix_cum(rec: np.ndarray) -> np.ndarray:
    pre = (rec[:, 1].astype(np.int64) << 16) | (rec[:, 2].astype(np.int64) << 8) | rec[:, 3]
    return np.cumsum(np.bincount(pre, minlength=1 << 24)).astype(np.int64)


def check_index(rec: np.ndarray, dig: dict) -> None:
    """Sorted records (reference layout, byte 0 = LCP) against a golden digest."""
    d = dig["index"]
    assert rec.shape == (d["count"], dig["rsize"])
    assert sha(canonical_rows(rec[:, 1:])) == d["records_multiset_sha"], "record multiset"
    assert sha(rec[:, 0]) == d["lcp_sha"], "LCP sequence"
    assert sha(rec[:, 1:11]) == d["kmer_sha"], "k-mer order"
    assert sha(prefix_cum(rec)) == d["cum_sha"], "prefix table"


def check_seeds(ns, cs, nb, cb, dig: dict) -> None:
    d = dig["seeds"]
    assert ns.shape[0] == d["n_count"] and cs.shape[0] == d["c_count"], "seed counts"
    assert sha(canonical_rows(ns)) == d["n_multiset_sha"], "N seed multiset"
    assert sha(canonical_rows(cs)) == d["c_multiset_sha"], "C seed multiset"
    assert list(nb) == d["nbuck"] and list(cb) == d["cbuck"], "seeds per A contig"


def check_diag(arr: np.ndarray, off: np.ndarray, unit: str, dig: dict) -> None:
    d = dig["diag"][unit]
    assert arr.shape == (d["count"], d["swide"])
    assert sha(arr) == d["sha"], "sorted diagonal panels (%s)" % unit
    assert np.diff(off).tolist() == d["panel"], "panel sizes (%s)" % unit


# ---- large cases: digests only (inputs regenerated, nothing stored) -----------

def check_index_large(rec: np.ndarray, dig: dict) -> None:
    d = dig["index"]
    assert rec.shape == (d["count"], dig["rsize"])
    assert multiset_digest(rec[:, 1:]) == d["records_multiset"], "record multiset"
    assert sha(rec[:, 0]) == d["lcp_sha"], "LCP sequence"
    assert sha(rec[:, 1:11]) == d["kmer_sha"], "k-mer order"
    assert sha(prefix_cum(rec)) == d["cum_sha"], "prefix table"


def check_seeds_large(ns, cs, nb, cb, dig: dict) -> None:
    d = dig["seeds"]
    assert ns.shape[0] == d["n_count"] and cs.shape[0] == d["c_count"], "seed counts"
    assert multiset_digest(ns) == d["n_multiset"], "N seed multiset"
    assert multiset_digest(cs) == d["c_multiset"], "C seed multiset"
    assert sha(np.asarray(nb, np.int64)) == d["nbuck_sha"] and sha(np.asarray(cb, np.int64)) == d["cbuck_sha"], \
        "seeds per A contig"


def check_diag_large(arr: np.ndarray, off: np.ndarray, unit: str, dig: dict) -> None:
    d = dig["diag"][unit]
    assert arr.shape == (d["count"], d["swide"])
    assert sha(arr) == d["sha"], "sorted diagonal panels (%s)" % unit
    assert sha(np.diff(off).astype(np.int64)) == d["panel_sha"], "panel sizes (%s)" % unit


def check_lines(lines, want: dict) -> None:
    got = lines_digest(lines, want["block"])
    assert got["count"] == want["count"], "alignment count %d, reference %d" % (got["count"], want["count"])
    if got["sha"] != want["sha"]:
        bad = [i for i, (x, y) in enumerate(zip(got["block_sha"], want["block_sha"])) if x != y]
        raise AssertionError("alignment stream differs from the reference's, first in lines %d-%d"
                             % (bad[0] * want["block"], (bad[0] + 1) * want["block"] - 1))
