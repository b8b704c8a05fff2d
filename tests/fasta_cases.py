"""Seeded FASTA texts for the GDB-ingest tests: the cases Create_GDB's reader
(lib/GDB.c:771-1057) treats specially, each as bytes.

``CASES`` maps a name to a builder; ``NTHR`` are the gap thresholds each case
is read with (0 is the reference's own setting, lib/GDB.c:1662).  ``ERRORS``
are texts the reference rejects.
"""
from __future__ import annotations

import numpy as np

NTHR = (0, 1, 4, 25)

_ACGT = np.frombuffer(b"ACGT", np.uint8)
_acgt = np.frombuffer(b"acgt", np.uint8)


def _bases(rng, n, lower=0.0):
    x = rng.integers(0, 4, n)
    s = np.where(rng.random(n) < lower, _acgt[x], _ACGT[x]).astype(np.uint8)
    return s


def _wrap(seq: bytes, widths, eol=b"\n") -> bytes:
    out, i, k = [], 0, 0
    while i < len(seq):
        w = widths[k % len(widths)]
        out.append(seq[i:i + w] + eol)
        i += w
        k += 1
    return b"".join(out)


def _with_runs(rng, n, nruns, maxrun, lower=0.0, lead=False, trail=False) -> bytes:
    """n characters with `nruns` N runs of length 1..maxrun (some lower case)."""
    s = bytearray(_bases(rng, n, lower).tobytes())
    for _ in range(nruns):
        L = int(rng.integers(1, maxrun + 1))
        p = int(rng.integers(0, max(1, n - L)))
        s[p:p + L] = (b"n" if rng.random() < 0.3 else b"N") * L
    if lead:
        s[:7] = b"NNNNNNN"
    if trail:
        s[-5:] = b"NNNNN"
    return bytes(s)


def case_single():
    return b">one\nACGT\n"


def case_widths():
    rng = np.random.default_rng(11)
    parts = []
    for k, w in enumerate(((1,), (60,), (80,), (1000,), (7, 13, 61), (4096,), (4095, 1))):
        seq = _bases(rng, int(rng.integers(200, 9000))).tobytes()
        parts.append(b">w%d\n" % k + _wrap(seq, w))
    return b"".join(parts)


def case_runs():
    rng = np.random.default_rng(12)
    parts = []
    for k in range(40):
        n = int(rng.integers(50, 3000))
        seq = _with_runs(rng, n, int(rng.integers(0, 12)), 30, lower=0.2, lead=k % 5 == 0, trail=k % 7 == 0)
        parts.append(b">r%d some description\n" % k + _wrap(seq, (int(rng.integers(1, 90)),)))
    return b"".join(parts)


def case_gap_lengths():
    # runs of every length around the thresholds, splitting contigs of every length mod 4
    parts = []
    rng = np.random.default_rng(13)
    for L in range(1, 30):
        seq = _bases(rng, 5 + L % 4).tobytes() + b"N" * L + _bases(rng, 9 + L % 3).tobytes()
        parts.append(b">g%d\n" % L + _wrap(seq, (6,)))
    return b"".join(parts)


def case_runs_across_lines():
    return (b">x\nACGTN\nNN\nNNNN\n\nNNAC\nGTNN\n>y\nNN\nN\nACGT\nTTTT\nN\n\nNN\n"
            b">z\nA\nN\nC\nNN\nG\n")


def case_crlf():
    rng = np.random.default_rng(14)
    seq = _with_runs(rng, 700, 4, 9)
    return b">crlf one\r\n" + _wrap(seq, (50,), b"\r\n") + b">crlf two\r\n" + _wrap(seq[:123], (40,), b"\r\n")


def case_blank_lines():
    return b">b\n\nACGTA\n\n\nNNNN\n\nCC\n\n>c\nG\n\n\n"


def case_headers():
    rng = np.random.default_rng(15)
    long = bytes(rng.integers(33, 127, 5000, dtype=np.uint8).tolist()).replace(b">", b"<")
    return (b">\nACGT\n"
            b">   spaced name\nAC\n"
            b">\ttabbed\tname \nGG\n"
            b"> \r\nTT\n"
            b">" + long + b"\nACGTACGT\n"
            b">x>y>z\nA\n")


def case_other_chars():
    # every printable character that is not N/n or '>' at a line start reads as a base
    body = bytes(c for c in range(32, 127) if c not in b"Nn")
    return b">odd\n" + body + b"\n" + b"RYKMSWBDHV-*.0123 ryk\n>tabs\n\tA\tC\t\n"


def case_many_scaffolds():
    rng = np.random.default_rng(16)
    parts = []
    for k in range(3000):
        n = int(rng.integers(1, 40))
        seq = _with_runs(rng, n, int(rng.integers(0, 2)), 3) if n > 4 else _bases(rng, n).tobytes()
        if seq.strip(b"Nn") == b"":
            seq = b"A" + seq
        parts.append(b">s%d\n" % k + _wrap(seq, (int(rng.integers(1, 20)),)))
    return b"".join(parts)


def case_scaffold_boundaries():
    # a scaffold that ends in N's followed by one that opens with N's
    return b">p\nACGTNNN\nNN\n>q\nNNNACGT\n>r\nNACGTN\n>s\nT\n"


def case_long_line():
    rng = np.random.default_rng(17)
    seq = _with_runs(rng, 200_000, 30, 200)
    return b">long\n" + seq + b"\n>after\n" + _wrap(seq[:5000], (70,))


CASES = {
    "single": case_single,
    "widths": case_widths,
    "runs": case_runs,
    "gap_lengths": case_gap_lengths,
    "runs_across_lines": case_runs_across_lines,
    "crlf": case_crlf,
    "blank_lines": case_blank_lines,
    "headers": case_headers,
    "other_chars": case_other_chars,
    "many_scaffolds": case_many_scaffolds,
    "scaffold_boundaries": case_scaffold_boundaries,
    "long_line": case_long_line,
}

ERRORS = {
    "empty": b"",
    "no_header": b"ACGT\n>a\nACGT\n",
    "no_final_newline": b">a\nACGT",
    "all_n": b">a\nACGT\n>b\nNNNN\nnn\n>c\nA\n",
    "empty_scaffold": b">a\nACGT\n>b\n>c\nA\n",
    "blank_scaffold": b">a\n\n\n>b\nAC\n",
    "last_empty": b">a\nACGT\n>b\n",
}


def random_fasta(seed: int, nbytes: int) -> bytes:
    """A large seeded FASTA of about `nbytes`: scaffolds of lognormal size with
    N runs and lower case, lines of 60-120 characters."""
    rng = np.random.default_rng(seed)
    parts, total, k = [], 0, 0
    while total < nbytes:
        n = int(min(nbytes - total + 100, max(100, rng.lognormal(11, 1.5))))
        s = np.frombuffer(_bases(rng, n, lower=0.1).tobytes(), np.uint8).copy()
        nr = int(rng.poisson(n / 20000)) + 1
        for _ in range(nr):
            L = int(rng.integers(1, 500))
            p = int(rng.integers(0, max(1, n - L)))
            s[p:p + L] = ord("N")
        if (s != ord("N")).sum() == 0:
            s[0] = ord("A")
        w = int(rng.integers(60, 121))
        body = _wrap(s.tobytes(), (w,))
        parts.append(b">scaffold_%d len=%d\n" % (k, n) + body)
        total += len(parts[-1])
        k += 1
    return b"".join(parts)
