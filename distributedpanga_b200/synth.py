"""Seeded synthetic genomes for the alignment path's workloads.

Bases are numeric 0..3 (A, C, G, T), as the GDB's NUMERIC form
(lib/GDB.h:77-81).  Both genomes go into ONE contig set -- A's contigs first,
then B's -- because the reference only implements FastGA's self mode: one GDB
holding every haplotype, every contig aligned against every contig
(src/pga-mpi-merge.c:57, SELF = 1).

Workloads (sizes in bases):

* ``small``  -- A = 2 Mbp uniform ACGT in contigs of U[50 kbp, 500 kbp];
  B = A + 5% substitutions + indels at 0.5% of positions (length U[1, 10])
  + 20 inverted segments of U[5 kbp, 50 kbp].
* ``chromset`` -- two 100 Mbp genomes at 40% GC, log-normal contig lengths
  (median 2 Mbp, sigma 1.0); 10% of A is 300 interspersed repeat families
  (unit U[300, 6000] bp, copies 10-20% diverged from their consensus);
  B = A at 1.5% substitutions, 0.2% indels (geometric length, mean 3),
  50 inversions and 50 translocations of U[10 kbp, 1 Mbp].

* ``full`` -- two 1 Gbp genomes built as ``small``: A uniform ACGT in contigs
  of U[50 kbp, 500 kbp], 40% of A overwritten by copies of 300 interspersed
  repeat families (unit U[300, 6000] bp, copies 10-20% diverged from their
  consensus) and 3% by tandem arrays (unit U[2, 200] bp, arrays of
  U[500, 10000] bp, copies 2% diverged); B = A at 2% substitutions, indels
  at 0.5% of positions (length U[1, 10]) and 20 inverted segments of
  U[5 kbp, 50 kbp].

``scale`` shrinks every length of a workload (genome size, contig and SV
lengths) by the same factor, for parity tests that must finish in seconds.
"""
from __future__ import annotations

import numpy as np

COMP = np.array([3, 2, 1, 0], dtype=np.uint8)


def revcomp(s: np.ndarray) -> np.ndarray:
    return COMP[s[::-1]]


def random_bases(rng: np.random.Generator, n: int, gc: float = 0.5) -> np.ndarray:
    at = (1.0 - gc) / 2.0
    p = np.array([at, gc / 2.0, gc / 2.0, at])
    return rng.choice(4, size=n, p=p).astype(np.uint8)


def substitute(rng: np.random.Generator, s: np.ndarray, rate: float) -> np.ndarray:
    out = s.copy()
    hit = rng.random(len(s)) < rate
    k = int(hit.sum())
    out[hit] = (out[hit] + rng.integers(1, 4, size=k).astype(np.uint8)) % 4
    return out


def indels(rng: np.random.Generator, s: np.ndarray, rate: float, lengths, gc: float) -> np.ndarray:
    """Insert or delete (50/50) at ``rate`` of positions; ``lengths(k)`` draws k lengths."""
    n = len(s)
    k = rng.binomial(n, rate)
    if k == 0:
        return s
    pos = np.sort(rng.choice(n, size=k, replace=False))
    lens = lengths(k)
    is_ins = rng.random(k) < 0.5
    pieces = []
    prev = 0
    for p, ln, ins in zip(pos.tolist(), lens.tolist(), is_ins.tolist()):
        if p < prev:
            continue
        pieces.append(s[prev:p])
        if ins:
            pieces.append(random_bases(rng, int(ln), gc))
            prev = p
        else:
            prev = min(n, p + int(ln))
    pieces.append(s[prev:])
    return np.concatenate(pieces)


def invert(rng: np.random.Generator, s: np.ndarray, count: int, lo: int, hi: int) -> np.ndarray:
    out = s.copy()
    n = len(out)
    for _ in range(count):
        ln = int(rng.integers(lo, hi + 1))
        if ln >= n:
            continue
        p = int(rng.integers(0, n - ln))
        out[p:p + ln] = revcomp(out[p:p + ln])
    return out


def translocate(rng: np.random.Generator, s: np.ndarray, count: int, lo: int, hi: int) -> np.ndarray:
    out = s
    for _ in range(count):
        n = len(out)
        ln = int(rng.integers(lo, hi + 1))
        if ln >= n // 2:
            continue
        p = int(rng.integers(0, n - ln))
        seg = out[p:p + ln]
        rest = np.concatenate([out[:p], out[p + ln:]])
        q = int(rng.integers(0, len(rest)))
        out = np.concatenate([rest[:q], seg, rest[q:]])
    return out


def split_uniform(rng: np.random.Generator, s: np.ndarray, lo: int, hi: int) -> list:
    out, p, n = [], 0, len(s)
    while p < n:
        ln = int(rng.integers(lo, hi + 1))
        if n - p - ln < lo:          # fold a short tail into the last contig
            ln = n - p
        out.append(s[p:p + ln])
        p += ln
    return out


def split_lognormal(rng: np.random.Generator, s: np.ndarray, median: float, sigma: float,
                    lo: int) -> list:
    out, p, n = [], 0, len(s)
    while p < n:
        ln = max(lo, int(rng.lognormal(np.log(median), sigma)))
        if n - p - ln < lo:
            ln = n - p
        out.append(s[p:p + ln])
        p += ln
    return out


def plant_repeats(rng: np.random.Generator, s: np.ndarray, fraction: float, families: int,
                  unit_lo: int, unit_hi: int, div_lo: float, div_hi: float, gc: float) -> np.ndarray:
    out = s.copy()
    n = len(out)
    cons = [random_bases(rng, int(rng.integers(unit_lo, unit_hi + 1)), gc) for _ in range(families)]
    target = int(fraction * n)
    covered = 0
    while covered < target:
        c = cons[int(rng.integers(0, families))]
        if len(c) >= n:
            break
        copy = substitute(rng, c, float(rng.uniform(div_lo, div_hi)))
        if rng.random() < 0.5:
            copy = revcomp(copy)
        p = int(rng.integers(0, n - len(copy)))
        out[p:p + len(copy)] = copy
        covered += len(copy)
    return out


def make_small(seed: int = 1, scale: float = 1.0) -> list:
    """A and B of the 2 Mbp workload, as one list of contigs (A's first)."""
    rng = np.random.default_rng(seed)
    g = int(2_000_000 * scale)
    a = random_bases(rng, g)
    b = substitute(rng, a, 0.05)
    b = indels(rng, b, 0.005, lambda k: rng.integers(1, 11, size=k), 0.5)
    b = invert(rng, b, 20, max(40, int(5_000 * scale)), max(80, int(50_000 * scale)))
    lo, hi = max(200, int(50_000 * scale)), max(400, int(500_000 * scale))
    return split_uniform(rng, a, lo, hi) + split_uniform(rng, b, lo, hi)


def make_chromset(seed: int = 2, scale: float = 1.0) -> list:
    """A and B of the 2 x 100 Mbp workload, as one list of contigs (A's first)."""
    rng = np.random.default_rng(seed)
    gc = 0.40
    g = int(100_000_000 * scale)
    a = random_bases(rng, g, gc)
    a = plant_repeats(rng, a, 0.10, 300, max(20, int(300 * min(1.0, scale * 10))),
                      max(40, int(6000 * min(1.0, scale * 10))), 0.10, 0.20, gc)
    b = substitute(rng, a, 0.015)
    b = indels(rng, b, 0.002, lambda k: rng.geometric(1.0 / 3.0, size=k), gc)
    svlo, svhi = max(50, int(10_000 * scale)), max(100, int(1_000_000 * scale))
    b = invert(rng, b, 50, svlo, svhi)
    b = translocate(rng, b, 50, svlo, svhi)
    med = max(2_000, 2_000_000 * scale)
    lo = max(100, int(10_000 * scale))
    return split_lognormal(rng, a, med, 1.0, lo) + split_lognormal(rng, b, med, 1.0, lo)


def plant_tandems(rng: np.random.Generator, s: np.ndarray, fraction: float, unit_lo: int, unit_hi: int,
                  arr_lo: int, arr_hi: int, div: float, gc: float) -> np.ndarray:
    """Overwrites ``fraction`` of s with tandem arrays: a random unit repeated
    to the array's length, then ``div`` of its bases substituted."""
    out = s.copy()
    n = len(out)
    target = int(fraction * n)
    covered = 0
    while covered < target:
        unit = random_bases(rng, int(rng.integers(unit_lo, unit_hi + 1)), gc)
        ln = int(rng.integers(arr_lo, arr_hi + 1))
        if ln >= n:
            break
        arr = substitute(rng, np.resize(unit, ln), div)
        p = int(rng.integers(0, n - ln))
        out[p:p + ln] = arr
        covered += ln
    return out


def make_full(seed: int = 3, scale: float = 1.0) -> list:
    """A and B of the 2 x 1 Gbp workload, as one list of contigs (A's first)."""
    rng = np.random.default_rng(seed)
    g = int(1_000_000_000 * scale)
    a = random_bases(rng, g)
    a = plant_repeats(rng, a, 0.40, 300, max(20, int(300 * min(1.0, scale * 10))),
                      max(40, int(6000 * min(1.0, scale * 10))), 0.10, 0.20, 0.5)
    a = plant_tandems(rng, a, 0.03, 2, 200, max(50, int(500 * min(1.0, scale * 10))),
                      max(100, int(10_000 * min(1.0, scale * 10))), 0.02, 0.5)
    b = substitute(rng, a, 0.02)
    b = indels(rng, b, 0.005, lambda k: rng.integers(1, 11, size=k), 0.5)
    b = invert(rng, b, 20, max(40, int(5_000 * scale)), max(80, int(50_000 * scale)))
    lo, hi = max(200, int(50_000 * scale)), max(400, int(500_000 * scale))
    return split_uniform(rng, a, lo, hi) + split_uniform(rng, b, lo, hi)


def make_pangenome(seed: int = 4, scale: float = 1.0) -> list:
    """The batched form's pan-genome: a 50 Mbp seeded reference (uniform ACGT)
    and 16 haplotypes of it, each with its own substitution rate in
    [0.1%, 1%], indels at a tenth of that (geometric length, mean 3), 10
    inversions and 5 translocations of U[1 kbp, 100 kbp]; every genome cut
    into log-normal contigs (median 224 kbp, sigma 1) kept within
    [10 kbp, 5 Mbp].  One contig list, the reference's first."""
    rng = np.random.default_rng(seed)
    g = int(50_000_000 * scale)
    ref = random_bases(rng, g)
    genomes = [ref]
    svlo, svhi = max(50, int(1_000 * scale)), max(100, int(100_000 * scale))
    for _ in range(16):
        d = float(rng.uniform(0.001, 0.01))
        h = substitute(rng, ref, d)
        h = indels(rng, h, d / 10, lambda k: rng.geometric(1.0 / 3.0, size=k), 0.5)
        h = invert(rng, h, 10, svlo, svhi)
        h = translocate(rng, h, 5, svlo, svhi)
        genomes.append(h)
    f = max(scale, 0.05)
    lo, hi, med = int(10_000 * f), int(5_000_000 * f), 224_000 * f
    out = []
    for s in genomes:
        p, n = 0, len(s)
        while p < n:
            ln = int(min(hi, max(lo, rng.lognormal(np.log(med), 1.0))))
            if n - p - ln < lo:
                ln = n - p
            out.append(s[p:p + ln])
            p += ln
    return out


def make_target(seed: int = 5, scale: float = 1.0) -> list:
    """The served form's resident target: one 1 Gbp genome built as A of
    ``chromset`` (40% GC, 10% in 300 repeat families, log-normal contigs of
    median 2 Mbp; below scale 0.05 the contig lengths stop shrinking)."""
    rng = np.random.default_rng(seed)
    gc = 0.40
    g = int(1_000_000_000 * scale)
    a = random_bases(rng, g, gc)
    a = plant_repeats(rng, a, 0.10, 300, max(20, int(300 * min(1.0, scale * 100))),
                      max(40, int(6000 * min(1.0, scale * 100))), 0.10, 0.20, gc)
    f = max(scale, 0.05)             # contig lengths shrink at most 20-fold
    return split_lognormal(rng, a, 2_000_000 * f, 1.0, int(10_000 * f))


def make_query(rng: np.random.Generator, target: list, size: int, divergence: float,
               median: float = 2_000_000) -> list:
    """A query assembly of ``size`` bases: a stretch of the target's
    concatenated contigs (a quarter of it reverse-complemented) with
    substitutions at ``divergence`` and indels (geometric length, mean 3) at a
    tenth of that, cut into log-normal contigs."""
    cat = np.concatenate(target)
    size = min(size, len(cat))
    p = int(rng.integers(0, len(cat) - size + 1))
    q = cat[p:p + size]
    if rng.random() < 0.25:
        q = revcomp(q)
    q = substitute(rng, q, divergence)
    q = indels(rng, q, divergence / 10, lambda k: rng.geometric(1.0 / 3.0, size=k), 0.40)
    return split_lognormal(rng, q, median, 1.0, max(100, min(10_000, size // 4)))


def query_stream(target: list, n: int, rate: float, size_lo: int, size_hi: int, seed: int = 11,
                 div_lo: float = 0.005, div_hi: float = 0.05, median: float = 2_000_000) -> list:
    """n requests of a Poisson stream (``rate`` per second): (arrival seconds,
    query contigs), sizes log-uniform in [size_lo, size_hi], divergence
    uniform in [div_lo, div_hi]."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate)) if rate > 0 else 0.0
        size = int(np.exp(rng.uniform(np.log(size_lo), np.log(size_hi))))
        out.append((t, make_query(rng, target, size, float(rng.uniform(div_lo, div_hi)), median)))
    return out


def fasta_bytes(contigs: list, prefix: str = "ctg", width: int = 80) -> bytes:
    """FASTA text of numeric contigs, named <prefix><i>."""
    letters = np.frombuffer(b"ACGT", dtype=np.uint8)
    parts = []
    for i, c in enumerate(contigs):
        s = letters[c].tobytes()
        parts.append(b">%s%d\n" % (prefix.encode(), i))
        parts.append(b"".join(s[j:j + width] + b"\n" for j in range(0, len(s), width)))
    return b"".join(parts)


WORKLOADS = {"small": make_small, "chromset": make_chromset, "full": make_full, "pangenome": make_pangenome}


def make(workload: str, seed: int | None = None, scale: float = 1.0) -> list:
    fn = WORKLOADS[workload]
    return fn(scale=scale) if seed is None else fn(seed=seed, scale=scale)


def write_fasta(path: str, contigs: list, width: int = 80) -> None:
    letters = np.frombuffer(b"ACGT", dtype=np.uint8)
    with open(path, "wb") as f:
        for i, c in enumerate(contigs):
            f.write(b">ctg%d\n" % i)
            s = letters[c].tobytes()
            for j in range(0, len(s), width):
                f.write(s[j:j + width])
                f.write(b"\n")
