"""ctypes binding of the C restatement (oracle/pga_oracle.c) and runners for
the reference pipeline compiled from source (oracle/_ref).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_LIB = None

i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_tmap.restype = C.POINTER(C.c_uint8)
        L.orc_tmap.argtypes = []
        L.orc_extract.restype = C.c_int64
        L.orc_extract.argtypes = [u8p, C.c_int, i64p, i64p, C.c_int, C.c_int, C.c_void_p, C.c_int64]
        L.orc_sort_records.restype = None
        L.orc_sort_records.argtypes = [u8p, C.c_int64, C.c_int]
        L.orc_lcp_bases.restype = C.c_int
        L.orc_lcp_bases.argtypes = [u8p, u8p]
        L.orc_build_adapter.restype = C.c_int64
        L.orc_build_adapter.argtypes = [u8p, C.c_int64, C.c_int, C.c_int, C.c_int, u8p, i64p]
        L.orc_merge.restype = C.c_int
        L.orc_merge.argtypes = [u8p, i64p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_void_p, C.c_int64, C.POINTER(C.c_int64),
                                C.c_void_p, C.c_int64, C.POINTER(C.c_int64), i64p, i64p]
        L.orc_reimport_sort.restype = C.c_int
        L.orc_reimport_sort.argtypes = [u8p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64,
                                        C.c_int, u8p, i64p]
        L.orc_fasta_gdb.restype = C.c_int
        L.orc_fasta_gdb.argtypes = [C.c_char_p, C.c_int64, C.c_int, i64p, C.c_int64, i64p, C.c_int64,
                                    u8p, C.c_int64, u8p, C.c_int64, i64p, i64p, C.c_char_p, C.c_int]
        _LIB = L
    return _LIB


def tmap() -> np.ndarray:
    p = lib().orc_tmap()
    return np.array([p[i] for i in range(256)], dtype=np.uint8)


def extract(cs, posb: int, ctgb: int) -> np.ndarray:
    """Records of every contig in the reference's emission order."""
    L = lib()
    rsize = 12 + posb + ctgb
    n = L.orc_extract(cs.bps, cs.ncontig, cs.clen, cs.boff, posb, ctgb, None, 0)
    out = np.zeros(max(1, n) * rsize, dtype=np.uint8)
    L.orc_extract(cs.bps, cs.ncontig, cs.clen, cs.boff, posb, ctgb, out.ctypes.data, n)
    return out[: n * rsize].reshape(n, rsize)


def sort_records(rec: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(rec.copy())
    lib().orc_sort_records(out.reshape(-1), out.shape[0], out.shape[1])
    return out


def build_adapter(rec: np.ndarray, posb: int, ctgb: int):
    n, rsize = rec.shape
    eb = 9 + posb + ctgb
    ent = np.zeros(max(1, n) * eb, dtype=np.uint8)
    cum = np.zeros(1 << 24, dtype=np.int64)
    big = lib().orc_build_adapter(np.ascontiguousarray(rec).reshape(-1), n, rsize, posb, ctgb, ent, cum)
    return ent[: n * eb].reshape(n, eb), cum, int(big)


def merge(ent: np.ndarray, cum: np.ndarray, posb: int, ctgb: int, freq: int, ncontig: int):
    """(N seeds, C seeds, nbuck, cbuck) -- seeds as (count, seed_bytes) uint8 arrays."""
    L = lib()
    n, eb = ent.shape
    sb = 1 + 2 * (posb + ctgb)
    nl, cl = C.c_int64(0), C.c_int64(0)
    nb = np.zeros(ncontig, dtype=np.int64)
    cb = np.zeros(ncontig, dtype=np.int64)
    flat = np.ascontiguousarray(ent).reshape(-1)
    if n == 0:
        flat = np.zeros(1, dtype=np.uint8)
    L.orc_merge(flat, cum, n, eb, posb, ctgb, freq, ncontig, None, 0, C.byref(nl), None, 0, C.byref(cl), nb, cb)
    ns = np.zeros(max(1, nl.value), dtype=np.uint8)
    css = np.zeros(max(1, cl.value), dtype=np.uint8)
    L.orc_merge(flat, cum, n, eb, posb, ctgb, freq, ncontig, ns.ctypes.data, nl.value, C.byref(nl),
                css.ctypes.data, cl.value, C.byref(cl), nb, cb)
    return ns[: nl.value].reshape(-1, sb), css[: cl.value].reshape(-1, sb), nb, cb


def reimport_sort(seeds: np.ndarray, posb: int, ctgb: int, comp: int, ncontig: int,
                  amxpos: int, dbyte: int):
    """(records (count, swide), panel offsets (ncontig+1))."""
    swide = 2 * dbyte + ctgb + 2
    ns = seeds.shape[0]
    out = np.zeros(max(1, ns) * swide, dtype=np.uint8)
    off = np.zeros(ncontig + 1, dtype=np.int64)
    flat = np.ascontiguousarray(seeds).reshape(-1)
    if ns == 0:
        flat = np.zeros(1, dtype=np.uint8)
    lib().orc_reimport_sort(flat, ns * seeds.shape[1] if ns else 0, posb, ctgb, comp, ncontig,
                            amxpos, dbyte, out, off)
    return out[: ns * swide].reshape(ns, swide), off


# ---- the reference pipeline compiled from source (oracle/_ref) -------------

def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, x))
               for x in ("pga-mpi-merge", "fa2gdb", "gdbdump", "GIXmake_dump", "ALNtoPAF"))


def fasta_gdb(text: bytes, nthr: int = 0) -> dict:
    """Create_GDB's FASTA reader on `text` (orc_fasta_gdb).  Raises ValueError
    with the reader's message for an input it rejects."""
    n = len(text)
    cap = n + 2
    scf = np.zeros(4 * cap, np.int64)
    ctg = np.zeros(4 * cap, np.int64)
    hdr = np.zeros(cap, np.uint8)
    bps = np.zeros(cap, np.uint8)
    sizes = np.zeros(6, np.int64)
    count = np.zeros(4, np.int64)
    err = C.create_string_buffer(256)
    r = lib().orc_fasta_gdb(text, n, nthr, scf, cap, ctg, cap, hdr, cap, bps, cap, sizes, count, err, 256)
    if r == -1:
        raise ValueError(err.value.decode())
    if r != 0:
        raise RuntimeError("orc_fasta_gdb: capacity")
    nscaff, ncontig, nbps, hdrtot, maxctg, seqtot = (int(x) for x in sizes)
    return {"nscaff": nscaff, "ncontig": ncontig, "maxctg": maxctg, "seqtot": seqtot,
            "scaffolds": scf[:4 * nscaff].reshape(-1, 4).copy(),
            "contigs": ctg[:4 * ncontig].reshape(-1, 4).copy(),
            "headers": hdr[:hdrtot].tobytes(), "bps": bps[:nbps].copy(), "count": count.copy()}


def ref_make_gdb(fasta: str, stem: str, nthr: int | None = None) -> None:
    cmd = [os.path.join(REF_DIR, "fa2gdb"), fasta, stem + ".1gdb"]
    if nthr is not None:
        cmd.append(str(nthr))
    subprocess.run(cmd, check=True, capture_output=True)


def ref_gdb_tables(stem: str) -> dict:
    """The GDB as the reference reads it back (gdbdump -s): contig rows
    (clen, boff, sbeg, scaf), scaffold rows (fctg, ectg, slen, hoff), the
    headers, the frequencies as floats and the .bps bytes."""
    out = subprocess.run([os.path.join(REF_DIR, "gdbdump"), "-s", stem], check=True,
                         capture_output=True).stdout.decode("latin-1").split("\n")
    head = out[0].split()
    ncontig = int(head[0])
    ctg = np.array([list(map(int, l.split())) for l in out[1:1 + ncontig]], np.int64).reshape(-1, 4)
    nscaff, hdrtot = (int(x) for x in out[1 + ncontig].split())
    scf, names = [], []
    for l in out[2 + ncontig:2 + ncontig + nscaff]:
        f = l.split(" ", 4)
        scf.append([int(x) for x in f[:4]])
        names.append(f[4] if len(f) > 4 else "")
    with open(head[7], "rb") as f:
        bps = np.frombuffer(f.read(), np.uint8)
    return {"ncontig": ncontig, "maxctg": int(head[1]), "seqtot": int(head[2]),
            "freq": np.array([float(x) for x in head[3:7]], np.float32),
            "contigs": ctg, "scaffolds": np.array(scf, np.int64).reshape(-1, 4),
            "names": names, "hdrtot": hdrtot, "bps": bps}


def ref_gdbdump(stem: str):
    out = subprocess.run([os.path.join(REF_DIR, "gdbdump"), stem], check=True,
                         capture_output=True, text=True).stdout.split("\n")
    head = out[0].split()
    rows = [list(map(int, l.split())) for l in out[1:] if l.strip()]
    return {"ncontig": int(head[0]), "maxctg": int(head[1]), "seqtot": int(head[2]),
            "freq": [float(x) for x in head[3:7]], "seqpath": head[7],
            "clen": [r[0] for r in rows], "boff": [r[1] for r in rows]}


def ref_run(stem: str, workdir: str, threads: int = 8, timeout: float = 3600.0,
            driver: str = "pga-mpi-merge") -> dict:
    """Build the .gix and run the reference's single-process pipeline on <stem>
    (`driver`: the stock build, or pga-mpi-merge-b200, the same driver linked
    with the B200 drop-in stages, which writes no dumps).

    Returns paths of its dumps: index.bin, seeds.bin and the .1aln."""
    dump = os.path.join(workdir, "dump")
    os.makedirs(dump, exist_ok=True)
    env = dict(os.environ)
    env["PATH"] = REF_DIR + os.pathsep + env.get("PATH", "")
    env["ORACLE_DUMP_DIR"] = dump
    env.setdefault("PGA_SCRATCH_DIR", "/tmp")
    # GIXmake_dump's own text dump of every k-mer is not read here
    env.setdefault("GIXMAKE_DUMP_PATH", os.devnull)
    with open(os.path.join(workdir, "gix.log"), "w") as log:
        subprocess.run([os.path.join(REF_DIR, "GIXmake_dump"), "-T%d" % threads, stem + ".1gdb"],
                       check=True, stdout=log, stderr=subprocess.STDOUT, cwd=workdir, env=env,
                       timeout=timeout)
    with open(os.path.join(workdir, "merge.log"), "w") as log:
        subprocess.run([os.path.join(REF_DIR, driver), stem], check=True, stdout=log,
                       stderr=subprocess.STDOUT, cwd=workdir, env=env, timeout=timeout)
    return {"index": os.path.join(dump, "index.bin"), "seeds": os.path.join(dump, "seeds.bin"),
            "aln": os.path.join(workdir, "out.rank0.paf"), "log": os.path.join(workdir, "merge.log")}


def read_index_dump(path: str):
    with open(path, "rb") as f:
        rsize, posb, ctgb = np.frombuffer(f.read(12), dtype=np.int32)
        n = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
        rec = np.frombuffer(f.read(n * int(rsize)), dtype=np.uint8).reshape(n, int(rsize))
    return rec, int(posb), int(ctgb)


def read_seed_dump(path: str):
    with open(path, "rb") as f:
        sb, nc = [int(x) for x in np.frombuffer(f.read(8), dtype=np.int32)]
        nl, cl = [int(x) for x in np.frombuffer(f.read(16), dtype=np.int64)]
        ns = np.frombuffer(f.read(nl), dtype=np.uint8).reshape(-1, sb)
        cs = np.frombuffer(f.read(cl), dtype=np.uint8).reshape(-1, sb)
        nb = np.frombuffer(f.read(8 * nc), dtype=np.int64)
        cb = np.frombuffer(f.read(8 * nc), dtype=np.int64)
    return ns, cs, nb, cb


def canonical_rows(a: np.ndarray) -> np.ndarray:
    """Rows of a 2-D uint8 array in lexicographic order (for multiset equality)."""
    if a.shape[0] == 0:
        return a
    v = np.ascontiguousarray(a).view(np.dtype((np.void, a.shape[1]))).reshape(-1)
    return a[np.argsort(v, kind="stable")]
