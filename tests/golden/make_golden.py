"""Generates the golden fixtures in tests/golden/ by running the reference.

For every case below this script builds a seeded contig set, writes it as
FASTA, and runs the reference's own single-process pipeline compiled from
source (oracle/_ref: fa2gdb -> GIXmake_dump -> pga-mpi-merge with dump
hooks -> alndump).  It stores

  <case>.npz         the inputs: .bps image, clen, boff, freq (and checks them
                     against the reference's own GDB: gdbdump + .bps bytes)
  <case>.json        digests of every stage's output: the index (record
                     multiset, LCP sequence, k-mer sequence, prefix table), the
                     N and C seed multisets and per-contig counts, the sorted
                     diagonal panels, and the .1aln record stream
  <case>.aln.txt.gz  the .1aln record stream itself (alndump text)

Large cases (LARGE below: the benchmarked 2 x 100 Mbp workload and a 20 Mbp
sample of the 2 x 1 Gbp generator) store only <case>.json, with
order-independent multiset digests (tests/helpers.py multiset_digest) in
place of sorted-row hashes, hashes of the per-contig arrays, and a hash per
block of 1000 alignments; their inputs are regenerated from the seeded
generator and pinned by input_sha.

Usage (needs oracle/_ref, i.e. `make -C oracle ref` with the reference tree
present):  python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

sys.path.insert(0, os.path.join(ROOT, "tests"))

from distributedpanga_b200 import gdb, synth  # noqa: E402
from helpers import lines_digest, multiset_digest  # noqa: E402
from oracle import binding as B  # noqa: E402


def rand(rng, n):
    return rng.integers(0, 4, size=n).astype(np.uint8)


def case_edge_mix():
    rng = np.random.default_rng(77)
    cs = []
    cs.append(np.zeros(6000, np.uint8))                        # poly-A: one huge prefix bucket
    cs.append(np.full(2500, 3, np.uint8))                      # poly-T
    cs.append(np.tile(np.array([0, 1], np.uint8), 1500))       # (AC)n tandem
    cs.append(np.tile(np.array([0, 1, 2], np.uint8), 800))     # (ACG)n tandem
    unit = rand(rng, 40)
    cs.append(np.tile(unit, 30))                               # 40-bp unit tandem
    for n in (11, 12, 13, 39, 40, 41, 67, 68, 256, 257):       # range edges (E-04/05/08/09, R-03)
        cs.append(rand(rng, n))
    base = rand(rng, 5000)
    cs.append(base)
    cs.append(synth.substitute(rng, base, 0.02))               # a diverged copy: seeds + alignments
    cs.append(synth.revcomp(synth.substitute(rng, base[1000:4000], 0.03)))
    return cs


def case_many_contigs():
    rng = np.random.default_rng(78)
    fam = rand(rng, 180)
    cs = []
    for i in range(300):
        n = int(rng.integers(100, 256))
        s = rand(rng, n)
        if i % 3 == 0 and n > 190:
            p = int(rng.integers(0, n - 180))
            s[p:p + 180] = synth.substitute(rng, fam, 0.03)
        cs.append(s)
    return cs


CASES = {
    "small_full": lambda: synth.make("small"),
    "small_s002": lambda: synth.make("small", scale=0.02),
    "chromset_s0005": lambda: synth.make("chromset", scale=0.0005),
    "edge_mix": case_edge_mix,
    "many_contigs": case_many_contigs,
}


# Cases whose inputs are regenerated from the seeded generator by the tests
# (input_sha pins them) instead of being stored.
REGENERATED = {"small_full"}

# Large cases: digests only (see the module docstring).  The reference's
# pipeline takes about 20 s (full_s001) and 3 min (chromset_full) here.
LARGE = {
    "chromset_full": lambda: synth.make("chromset"),
    "full_s001": lambda: synth.make("full", scale=0.01),
    "pangenome_s002": lambda: synth.make("pangenome", scale=0.02),
}


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def run_case(name: str) -> None:
    large = name in LARGE
    contigs = LARGE[name]() if large else CASES[name]()
    cs = gdb.from_contigs(contigs)
    posb, ctgb, rsize = gdb.record_sizing(cs)
    dbyte, swide = gdb.diag_sizing(cs, ctgb)
    with tempfile.TemporaryDirectory() as tmp:
        fa = os.path.join(tmp, "g.fa")
        stem = os.path.join(tmp, "g")
        synth.write_fasta(fa, contigs)
        B.ref_make_gdb(fa, stem)
        d = B.ref_gdbdump(stem)
        assert d["clen"] == cs.clen.tolist() and d["boff"] == cs.boff.tolist(), "contig table"
        assert np.allclose(d["freq"], cs.freq, rtol=0, atol=1e-7), "freq"
        bps = np.fromfile(os.path.join(tmp, ".g.bps"), dtype=np.uint8)
        assert np.array_equal(bps, cs.bps), ".bps image"
        out = B.ref_run(stem, tmp)
        rec, rp, rc = B.read_index_dump(out["index"])
        assert (rp, rc, rec.shape[1]) == (posb, ctgb, rsize)
        ns, css, nb, cb = B.read_seed_dump(out["seeds"])
        diag = {}
        for u in ("N", "C"):
            p = os.path.join(tmp, "dump", "diag_%s.bin" % u)
            if os.path.exists(p):
                with open(p, "rb") as f:
                    sw, npart = [int(x) for x in np.frombuffer(f.read(8), np.int32)]
                    nel = int(np.frombuffer(f.read(8), np.int64)[0])
                    arr = np.frombuffer(f.read(nel * sw), np.uint8).reshape(nel, sw)
                    panel = np.frombuffer(f.read(8 * npart), np.int64) // sw
                diag[u] = {"swide": sw, "count": nel, "sha": sha(arr), "panel": panel.tolist()}
            else:
                panel = np.zeros(cs.ncontig, np.int64)
                diag[u] = {"swide": swide, "count": 0, "sha": sha(np.zeros((0, swide), np.uint8)),
                           "panel": [0] * cs.ncontig}
            if large:
                diag[u]["panel_sha"] = sha(np.asarray(panel, np.int64))
                del diag[u]["panel"]
        aln = subprocess.run([os.path.join(B.REF_DIR, "alndump"), out["aln"]], check=True,
                             capture_output=True, text=True).stdout
        with open(stem + ".gix", "rb") as f:
            f.seek(4 * 4 + 8 * (1 << 24) + 4 * 3 + 8 + 4 * 2)
            gix_perm = np.frombuffer(f.read(4 * cs.ncontig), np.int32).tolist()
    lines = [l for l in aln.split("\n") if l and not l.startswith("#")]
    if large:
        write_large(name, cs, posb, ctgb, rsize, dbyte, swide, rec, ns, css, nb, cb, diag, lines, gix_perm)
        return
    pre = (rec[:, 1].astype(np.int64) << 16) | (rec[:, 2].astype(np.int64) << 8) | rec[:, 3]
    cum = np.cumsum(np.bincount(pre, minlength=1 << 24)).astype(np.int64) if len(rec) else np.zeros(1 << 24, np.int64)
    dig = {
        "case": name,
        "ncontig": cs.ncontig, "maxctg": cs.maxctg, "seqtot": cs.seqtot,
        "posb": posb, "ctgb": ctgb, "rsize": rsize, "dbyte": dbyte, "swide": swide, "freq_cutoff": 10,
        "input_sha": sha(cs.bps) + sha(cs.clen) + sha(cs.boff),
        "index": {"count": int(rec.shape[0]),
                  "records_multiset_sha": sha(B.canonical_rows(rec[:, 1:])),
                  "lcp_sha": sha(rec[:, 0]), "kmer_sha": sha(rec[:, 1:11]), "cum_sha": sha(cum)},
        "seeds": {"seed_bytes": int(ns.shape[1]) if ns.size else 1 + 2 * (posb + ctgb),
                  "n_count": int(ns.shape[0]), "c_count": int(css.shape[0]),
                  "n_multiset_sha": sha(B.canonical_rows(ns)), "c_multiset_sha": sha(B.canonical_rows(css)),
                  "nbuck": nb.tolist(), "cbuck": cb.tolist()},
        "diag": diag,
        "aln": {"count": len(lines), "sha": hashlib.sha256("\n".join(lines).encode()).hexdigest()},
        "gix_perm": gix_perm,
    }
    if name not in REGENERATED:
        np.savez_compressed(os.path.join(HERE, name + ".npz"), bps=cs.bps, clen=cs.clen, boff=cs.boff,
                            freq=cs.freq)
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(dig, f, indent=1)
    with gzip.open(os.path.join(HERE, name + ".aln.txt.gz"), "wt") as f:
        f.write("\n".join(lines) + "\n")
    print(name, cs.ncontig, cs.seqtot, "records", rec.shape[0], "seeds", ns.shape[0], css.shape[0],
          "aln", len(lines))


def write_large(name, cs, posb, ctgb, rsize, dbyte, swide, rec, ns, css, nb, cb, diag, lines, gix_perm):
    from helpers import prefix_cum
    norm = [" ".join(l.split()) for l in lines]
    dig = {
        "case": name, "large": True,
        "ncontig": cs.ncontig, "maxctg": cs.maxctg, "seqtot": cs.seqtot,
        "posb": posb, "ctgb": ctgb, "rsize": rsize, "dbyte": dbyte, "swide": swide, "freq_cutoff": 10,
        "input_sha": sha(cs.bps) + sha(cs.clen) + sha(cs.boff),
        "index": {"count": int(rec.shape[0]), "records_multiset": multiset_digest(rec[:, 1:]),
                  "lcp_sha": sha(rec[:, 0]), "kmer_sha": sha(rec[:, 1:11]),
                  "cum_sha": sha(prefix_cum(rec)) if len(rec) else sha(np.zeros(1 << 24, np.int64))},
        "seeds": {"seed_bytes": 1 + 2 * (posb + ctgb), "n_count": int(ns.shape[0]), "c_count": int(css.shape[0]),
                  "n_multiset": multiset_digest(ns), "c_multiset": multiset_digest(css),
                  "nbuck_sha": sha(np.asarray(nb, np.int64)), "cbuck_sha": sha(np.asarray(cb, np.int64))},
        "diag": diag,
        "aln": lines_digest(norm),
        "aligned_bases": int(sum(int(l.split()[2]) - int(l.split()[1]) for l in norm)),
        "gix_perm_sha": sha(np.asarray(gix_perm, np.int32)),
    }
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(dig, f, indent=1)
    print(name, cs.ncontig, cs.seqtot, "records", rec.shape[0], "seeds", ns.shape[0], css.shape[0],
          "aln", len(lines))


if __name__ == "__main__":
    if not B.ref_available():
        sys.exit("oracle/_ref is not built: make -C oracle ref")
    for n in (sys.argv[1:] or list(CASES) + list(LARGE)):
        run_case(n)
