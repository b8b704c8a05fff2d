"""Digest helpers shared by the oracle and GPU parity tests."""
import hashlib

import numpy as np


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


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
