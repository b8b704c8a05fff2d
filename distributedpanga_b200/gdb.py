"""In-memory GDB: the contig table and 2-bit sequence the alignment path reads.

The reference reads a FastGA GDB (lib/GDB.h:45-70): a ``.1gdb`` ONE file with
the scaffold/contig table and base frequencies, plus a hidden ``.bps`` file
holding every contig 2-bit packed, four bases per byte with base i in bits
2*(i%4) (LSB first, lib/gene_core.c:336-378), each contig starting on a byte
boundary at ``boff`` (contigs are laid out back to back).  Extraction reads
only ``clen``, ``boff``, ``maxctg``, ``ncontig`` and the ``.bps`` bytes
(src/extract.c:85-249, src/record.c:18-37), so that is what this holds.

``freq`` is computed as the reference does when it creates a GDB
(lib/GDB.c:1083-1086, stored as float): the fraction of each base over all
contigs.  It feeds the aligner's scoring tables (lib/align.c:222-268).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class ContigSet:
    bps: np.ndarray        # uint8, the .bps image
    clen: np.ndarray       # int64 per contig
    boff: np.ndarray       # int64 per contig, byte offset into bps
    freq: np.ndarray       # float32[4], A C G T

    @property
    def ncontig(self) -> int:
        return int(len(self.clen))

    @property
    def maxctg(self) -> int:
        return int(self.clen.max()) if len(self.clen) else 0

    @property
    def seqtot(self) -> int:
        return int(self.clen.sum())

    def contig(self, r: int) -> np.ndarray:
        """Contig r as NUMERIC bases (0..3)."""
        n = int(self.clen[r])
        b = self.bps[int(self.boff[r]): int(self.boff[r]) + (n + 3) // 4]
        out = np.empty(len(b) * 4, dtype=np.uint8)
        for k in range(4):
            out[k::4] = (b >> (2 * k)) & 3
        return out[:n]


def pack_contig(s: np.ndarray) -> np.ndarray:
    """2-bit pack NUMERIC bases LSB-first, four per byte (lib/gene_core.c:336-357)."""
    n = len(s)
    pad = (-n) % 4
    t = np.concatenate([s.astype(np.uint8), np.zeros(pad, dtype=np.uint8)]).reshape(-1, 4)
    return (t[:, 0] | (t[:, 1] << 2) | (t[:, 2] << 4) | (t[:, 3] << 6)).astype(np.uint8)


def from_contigs(contigs: list) -> ContigSet:
    clen = np.array([len(c) for c in contigs], dtype=np.int64)
    nbytes = (clen + 3) // 4
    boff = np.zeros(len(contigs), dtype=np.int64)
    if len(contigs) > 1:
        boff[1:] = np.cumsum(nbytes)[:-1]
    bps = np.concatenate([pack_contig(c) for c in contigs]) if contigs else np.zeros(0, np.uint8)
    counts = np.zeros(4, dtype=np.int64)
    for c in contigs:
        counts += np.bincount(c, minlength=4)[:4]
    tot = max(1, int(clen.sum()))
    freq = np.array([counts[i] / tot for i in range(4)], dtype=np.float32)
    return ContigSet(bps=bps, clen=clen, boff=boff, freq=freq)


def record_sizing(cs: ContigSet) -> tuple:
    """(position bytes, contig|strand bytes, record bytes) as src/record.c:18-37."""
    def inclusive(v: int) -> int:
        b, cum = 0, 1
        while cum < v + 1:
            cum *= 256
            b += 1
        return b
    posb = inclusive(cs.maxctg)
    ctgb = inclusive(2 * cs.ncontig - 1)
    return posb, ctgb, 1 + 10 + 1 + posb + ctgb


def diag_sizing(cs: ContigSet, ctgb: int) -> tuple:
    """(DBYTE, swide) as src/pga-mpi-merge.c:415-425 and src/fastga_pipeline.c:1736."""
    maxdag = 2 * cs.maxctg
    d, cum = 0, 1
    while cum < maxdag:
        cum *= 256
        d += 1
    return d, 2 * d + ctgb + 2
