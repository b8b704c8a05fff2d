"""Generates tests/golden/fasta_edge.npz: the GDBs the reference builds from
the FASTA texts of tests/fasta_cases.py.

For every case and gap threshold it runs the reference's own Create_GDB /
Write_GDB (oracle/_ref/fa2gdb, lib/GDB.c:442,1519) and reads the result back
with its Read_GDB (oracle/_ref/gdbdump -s, lib/GDB.c:1171).  Stored per
"<case>.<nthr>":
  .text_sha   sha256 of the FASTA text (guards against generator drift)
  .contigs    ncontig x {clen, boff, sbeg, scaf}
  .scaffolds  nscaff x {fctg, ectg, slen, hoff}
  .names      the scaffold names, each ended by NUL
  .freq       GDB.freq (float32)
  .bps_sha    sha256 of the .bps file
and per error case "<name>.rejected" = 1 when fa2gdb refuses the text.

Usage (needs oracle/_ref):  python tests/golden/make_fasta_golden.py
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import fasta_cases as FC  # noqa: E402
from oracle import binding as B  # noqa: E402


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def reference_gdb(text: bytes, nthr: int, work: str):
    fa = os.path.join(work, "in.fa")
    with open(fa, "wb") as f:
        f.write(text)
    stem = os.path.join(work, "g")
    try:
        B.ref_make_gdb(fa, stem, nthr)
    except subprocess.CalledProcessError:
        return None
    return B.ref_gdb_tables(stem)


def main() -> None:
    out = {}
    with tempfile.TemporaryDirectory() as work:
        for name, build in FC.CASES.items():
            text = build()
            for nthr in FC.NTHR:
                r = reference_gdb(text, nthr, work)
                assert r is not None, (name, nthr)
                k = "%s.%d." % (name, nthr)
                out[k + "text_sha"] = np.array(sha(text))
                out[k + "contigs"] = r["contigs"]
                out[k + "scaffolds"] = r["scaffolds"]
                out[k + "names"] = np.frombuffer(b"".join(n.encode("latin-1") + b"\0" for n in r["names"]),
                                                 np.uint8)
                out[k + "freq"] = r["freq"]
                out[k + "bps_sha"] = np.array(sha(r["bps"].tobytes()))
        for name, text in FC.ERRORS.items():
            out[name + ".rejected"] = np.array(reference_gdb(text, 0, work) is None)
    np.savez_compressed(os.path.join(HERE, "fasta_edge.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
