"""Host-side mirror of the reference's stage interfaces over the C ABI.

Function names follow the reference's entry points for this path and take
and return its byte formats, as numpy arrays:

  extract_to_records     src/extract.h:40
  sort_records           src/sort.h:10  (with recalc_all_lcps: run_stage2 at world size 1)
  build_kmer_adapter     src/kmer_adapter.h:46
  self_adaptamer_merge   src/fastga_pipeline.h:18
  reimport_sort          reimport_thread + rmsd_sort, src/fastga_pipeline.c:1391, lib/RSDsort.c:292

``Device`` additionally keeps a GDB resident in HBM and runs the stages
without host round trips (``index_build`` -> ``merge`` -> ``diag_sort``).

There is no CPU fallback: every call goes to libpga_b200.so on a CUDA device,
and loading fails loudly when the library or the GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import gdb as _gdb

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpga_b200.so")

PGA_OK = 0
_ERRNAMES = {1: "CUDA error", 2: "bad argument", 3: "out of memory", 4: "beyond limits"}

i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
vp = C.c_void_p

_SIGS = {
    "pga_ctx_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
    "pga_ctx_destroy": (None, [vp]),
    "pga_last_error": (C.c_char_p, [vp]),
    "pga_ctx_set_stream": (C.c_int, [vp, vp]),
    "pga_ctx_synchronize": (C.c_int, [vp]),
    "pga_kernel_launches": (C.c_int64, [vp]),
    "pga_ctx_enable_timing": (C.c_int, [vp, C.c_int]),
    "pga_stage_times": (C.c_int, [vp, C.POINTER(C.c_float)]),
    "pga_alloc_times": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "pga_gdb_load": (C.c_int, [vp, u8p, C.c_int64, C.c_int, i64p, i64p]),
    "pga_record_sizing": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "pga_extract_to_records": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_uint8)),
                                         C.POINTER(C.c_int64)]),
    "pga_sort_records": (C.c_int, [vp, vp, C.c_int64, C.c_int, C.c_int]),
    "pga_build_kmer_adapter": (C.c_int, [vp, vp, C.c_int64, C.c_int, C.c_int, vp, i64p,
                                         C.POINTER(C.c_int64)]),
    "pga_self_adaptamer_merge": (C.c_int, [vp, vp, i64p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_int64),
                                           C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_int64),
                                           i64p, i64p]),
    "pga_reimport_sort": (C.c_int, [vp, vp, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64,
                                    C.c_int, vp, i64p]),
    "pga_index_build": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int64)]),
    "pga_index_copy_records": (C.c_int, [vp, vp]),
    "pga_index_copy_entries": (C.c_int, [vp, vp, vp, C.POINTER(C.c_int64)]),
    "pga_merge": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "pga_seeds_copy": (C.c_int, [vp, C.c_int, vp, vp]),
    "pga_seeds_load": (C.c_int, [vp, C.c_int, vp, C.c_int64]),
    "pga_diag_sort": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
    "pga_diag_copy": (C.c_int, [vp, C.c_int, vp, vp]),
    "pga_gdb_set_freq": (C.c_int, [vp, vp]),
    "pga_align": (C.c_int, [vp, C.POINTER(C.c_int64)]),
    "pga_align_copy": (C.c_int, [vp, vp, vp, vp]),
    "pga_align_stats": (C.c_int, [vp, vp]),
    "pga_align_set_ranges": (C.c_int, [vp, C.c_int64]),
    "pga_align_set_build": (C.c_int, [vp, C.c_int]),
    "pga_align_set_long_waves": (C.c_int, [vp, C.c_int]),
    "pga_index_set_digit_bits": (C.c_int, [vp, C.c_int]),
    "pga_align_times": (C.c_int, [vp, C.POINTER(C.c_float)]),
    "pga_align_work": (C.c_int, [vp, vp]),
    "pga_align_profile": (C.c_int, [vp, vp]),
    "pga_local_alignment": (C.c_int, [vp, C.c_int64, vp, C.POINTER(C.c_int64)]),
    "pga_local_alignment_copy": (C.c_int, [vp, vp, vp, vp]),
    "pga_write_1aln": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int,
                                 C.c_int, vp, vp, vp, vp, vp, C.c_int64, vp, vp, vp]),
    "pga_align_write_1aln": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                                       C.c_char_p, C.c_int, vp, vp, vp, vp]),
    "pga_read_gix": (C.c_int, [C.c_char_p, vp, vp, C.c_int64, vp, vp, vp, vp, C.c_int64]),
    "pga_fastga_ranges": (C.c_int, [C.c_int, vp, C.c_int64, vp, C.c_int64, C.c_int, vp]),
    "pga_write_1aln_binary": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                                        C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_int64, vp, vp, vp]),
    "pga_align_write_1aln_binary": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p,
                                              C.c_char_p, C.c_int, vp, vp, vp, vp]),
    "pga_reimport_sort_noalloc": (C.c_int, [vp, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64,
                                            C.c_int, vp, vp, vp]),
    "pga_gdb_ingest_fasta": (C.c_int, [vp, C.c_char_p, C.c_int64, C.c_int, vp]),
    "pga_index_write_gix": (C.c_int, [vp, C.c_char_p, C.c_int]),
    "pga_write_gix": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, C.c_int64, C.c_int64, vp]),
    "pga_gdb_copy": (C.c_int, [vp, vp, vp, vp, vp, vp]),
    "pga_gdb_ingest_times": (C.c_int, [vp, C.POINTER(C.c_float)]),
    "pga_gdb_write": (C.c_int, [vp, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p]),
    "pga_write_1gdb": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, vp, C.c_int, vp,
                                 vp, C.c_int64, C.c_int, vp, vp, C.c_int64]),
    "pga_target_create": (C.c_int, [vp, C.POINTER(vp)]),
    "pga_target_create_reuse": (C.c_int, [vp, C.c_int, C.POINTER(vp)]),
    "pga_align_reuse_stats": (C.c_int, [vp, vp]),
    "pga_target_destroy": (None, [vp]),
    "pga_target_info": (C.c_int, [vp, vp]),
    "pga_serve_load": (C.c_int, [vp, vp, C.c_char_p, C.c_int64, C.c_int, vp, vp]),
}

_LIB = None


def load_library():
    """The C-ABI library; raises if it is not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libpga_b200.so is not built (run distributedpanga_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L.free_ptr = C.CDLL(None).free
        L.free_ptr.argtypes = [vp]
        L.free_ptr.restype = None
        _LIB = L
    return _LIB


class PgaError(RuntimeError):
    pass


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(vp) if a.size else None


def _take(L, p, nbytes: int) -> np.ndarray:
    """Copy a malloc'd C buffer into numpy and free it."""
    out = np.empty(nbytes, dtype=np.uint8)
    if nbytes:
        C.memmove(out.ctypes.data, p, nbytes)
    if p:
        L.free_ptr(C.cast(p, vp))
    return out


# pga_stage_times' slots
STAGE_NAMES = ["extract_hist", "prefix_scan", "extract_scatter", "bucket_sort", "lcp", "entries_prefix_table",
               "merge", "diag_sort_n", "align", "diag_sort_c"]

class Device:
    """One pga_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        self.L = load_library()
        h = vp()
        rc = self.L.pga_ctx_create(device, C.byref(h))
        if rc != PGA_OK:
            raise PgaError("pga_ctx_create(%d) failed: %s" % (device, _ERRNAMES.get(rc, rc)))
        self.h = h
        self.cs = None
        self.ncontig = 0

    def close(self):
        if self.h:
            self.L.pga_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, what: str):
        if rc != PGA_OK:
            msg = self.L.pga_last_error(self.h)
            raise PgaError("%s: %s: %s" % (what, _ERRNAMES.get(rc, rc), msg.decode() if msg else ""))

    # ---- plumbing --------------------------------------------------------
    def set_stream(self, stream_handle: int | None):
        self._ck(self.L.pga_ctx_set_stream(self.h, stream_handle or None), "set_stream")

    def synchronize(self):
        self._ck(self.L.pga_ctx_synchronize(self.h), "synchronize")

    def launches(self) -> int:
        return int(self.L.pga_kernel_launches(self.h))

    def enable_timing(self, on: bool = True):
        self._ck(self.L.pga_ctx_enable_timing(self.h, 1 if on else 0), "enable_timing")

    def stage_times(self) -> dict:
        a = (C.c_float * 10)()
        self._ck(self.L.pga_stage_times(self.h, a), "stage_times")
        return dict(zip(STAGE_NAMES, [float(x) for x in a]))

    def alloc_times(self) -> dict:
        """Host ms inside cudaMalloc / cudaFree per stage (key "other":
        outside every stage) since timing was enabled, the number of those
        driver calls ("calls"), the bytes the context's arena holds
        ("held_bytes", "free_bytes") and how often the alignment buffers were
        freed to make room ("sheds")."""
        a = (C.c_double * 11)()
        n = (C.c_int64 * 4)()
        self._ck(self.L.pga_alloc_times(self.h, a, n), "alloc_times")
        d = dict(zip(STAGE_NAMES + ["other"], [float(x) for x in a]))
        d.update(calls=int(n[0]), held_bytes=int(n[1]), free_bytes=int(n[2]), sheds=int(n[3]))
        return d

    # ---- GDB -------------------------------------------------------------
    def gdb_load(self, cs: _gdb.ContigSet):
        bps = np.ascontiguousarray(cs.bps, dtype=np.uint8)
        if bps.size == 0:
            bps = np.zeros(1, dtype=np.uint8)
        self._ck(self.L.pga_gdb_load(self.h, bps, int(cs.bps.size), cs.ncontig,
                                     np.ascontiguousarray(cs.clen, dtype=np.int64),
                                     np.ascontiguousarray(cs.boff, dtype=np.int64)), "gdb_load")
        self.cs = cs
        self.ncontig = cs.ncontig

    def gdb_ingest_fasta(self, text, nthr: int = 0, nbytes: int | None = None, tables: bool = True):
        """Create_GDB (lib/GDB.c:442) of a FASTA text, parsed on the device;
        the result becomes this context's GDB (as gdb_load would leave it).
        `text` is bytes, or a host address with `nbytes` (pinned memory
        uploads fastest).  Returns the GdbTables, or with tables=False only
        the sizes {nscaff, ncontig, bps bytes, header bytes, maxctg, seqtot}."""
        if isinstance(text, int):
            ptr, n = C.cast(text, C.c_char_p), int(nbytes)
        else:
            text = bytes(text)
            ptr, n = text, len(text)
        sizes = np.zeros(6, dtype=np.int64)
        self._ck(self.L.pga_gdb_ingest_fasta(self.h, ptr, n, int(nthr), sizes.ctypes.data_as(vp)),
                 "gdb_ingest_fasta")
        self.cs = None
        self.ncontig = int(sizes[1])
        if not tables:
            return sizes
        t = self.gdb_tables(sizes)
        self.cs = _gdb.ContigSet(bps=t.bps, clen=t.contigs[:, 0].copy(), boff=t.contigs[:, 1].copy(),
                                 freq=t.freq)
        return t

    def serve_load(self, target: "Target", query, want_entries: bool = False, tables: bool = False):
        """One request against a resident target (pga_serve_load): this
        context's GDB becomes GDB(target text + query text) and its index is
        built by merging the query's sorted records into the target's.
        Returns the combined GDB's sizes (or its GdbTables) and sets nrec."""
        query = bytes(query)
        sizes = np.zeros(6, dtype=np.int64)
        n = C.c_int64()
        self._ck(self.L.pga_serve_load(self.h, target.h, query, len(query), 1 if want_entries else 0,
                                       sizes.ctypes.data_as(vp), C.byref(n)), "serve_load")
        self.nrec = n.value
        self.cs = None
        self.ncontig = int(sizes[1])
        if not tables:
            return sizes
        t = self.gdb_tables(sizes)
        self.cs = _gdb.ContigSet(bps=t.bps, clen=t.contigs[:, 0].copy(), boff=t.contigs[:, 1].copy(),
                                 freq=t.freq)
        return t

    def gdb_tables(self, sizes) -> "GdbTables":
        nscaff, ncontig, nbps, hdrtot = (int(x) for x in sizes[:4])
        bps = np.zeros(max(nbps, 1), dtype=np.uint8)
        ctg = np.zeros((ncontig, 4), dtype=np.int64)
        scf = np.zeros((nscaff, 4), dtype=np.int64)
        hdr = np.zeros(max(hdrtot, 1), dtype=np.uint8)
        cnt = np.zeros(4, dtype=np.int64)
        self._ck(self.L.pga_gdb_copy(self.h, bps.ctypes.data_as(vp), ctg.ctypes.data_as(vp),
                                     scf.ctypes.data_as(vp), hdr.ctypes.data_as(vp), cnt.ctypes.data_as(vp)),
                 "gdb_copy")
        return GdbTables(bps=bps[:nbps], contigs=ctg, scaffolds=scf, headers=hdr[:hdrtot].tobytes(), count=cnt,
                         maxctg=int(sizes[4]))

    def gdb_ingest_times(self) -> dict:
        a = (C.c_float * 2)()
        self._ck(self.L.pga_gdb_ingest_times(self.h, a), "gdb_ingest_times")
        return {"upload_ms": float(a[0]), "parse_ms": float(a[1])}

    def gdb_write(self, tpath: str, srcpath: str, command: str = "distributedpanga_b200"):
        """Write_GDB (lib/GDB.c:1519) of the ingested GDB: tpath and its .bps."""
        self._ck(self.L.pga_gdb_write(self.h, tpath.encode(), _PROG, _VERSION, command.encode(),
                                      srcpath.encode()), "gdb_write")

    def index_write_gix(self, stem: str, nparts: int = 8):
        """GIXmake's .gix + .ktab parts of the index built with entries."""
        self._ck(self.L.pga_index_write_gix(self.h, stem.encode(), int(nparts)), "index_write_gix")

    def record_sizing(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._ck(self.L.pga_record_sizing(self.h, C.byref(a), C.byref(b), C.byref(c)), "record_sizing")
        return a.value, b.value, c.value

    # ---- drop-in stages ----------------------------------------------------
    def extract_to_records(self, num_workers: int = 1, worker_id: int = 0) -> np.ndarray:
        p = C.POINTER(C.c_uint8)()
        n = C.c_int64()
        self._ck(self.L.pga_extract_to_records(self.h, num_workers, worker_id, C.byref(p), C.byref(n)),
                 "extract_to_records")
        rs = self.record_sizing()[2]
        return _take(self.L, p, n.value * rs).reshape(n.value, rs)

    def sort_records(self, rec: np.ndarray, posb: int, ctgb: int) -> np.ndarray:
        out = np.ascontiguousarray(rec, dtype=np.uint8).copy()
        self._ck(self.L.pga_sort_records(self.h, _ptr(out), out.shape[0], posb, ctgb), "sort_records")
        return out

    def build_kmer_adapter(self, rec: np.ndarray, posb: int, ctgb: int):
        rec = np.ascontiguousarray(rec, dtype=np.uint8)
        n = rec.shape[0]
        eb = 9 + posb + ctgb
        ent = np.zeros((n, eb), dtype=np.uint8)
        cum = np.zeros(1 << 24, dtype=np.int64)
        big = C.c_int64()
        self._ck(self.L.pga_build_kmer_adapter(self.h, _ptr(rec), n, posb, ctgb, _ptr(ent), cum,
                                               C.byref(big)), "build_kmer_adapter")
        return ent, cum, big.value

    def self_adaptamer_merge(self, ent: np.ndarray, cum: np.ndarray, posb: int, ctgb: int,
                             freq: int, ncontig: int):
        ent = np.ascontiguousarray(ent, dtype=np.uint8)
        pn, pc = C.POINTER(C.c_uint8)(), C.POINTER(C.c_uint8)()
        nl, cl = C.c_int64(), C.c_int64()
        nb = np.zeros(ncontig, dtype=np.int64)
        cb = np.zeros(ncontig, dtype=np.int64)
        self._ck(self.L.pga_self_adaptamer_merge(self.h, _ptr(ent), np.ascontiguousarray(cum, dtype=np.int64),
                                                 ent.shape[0], posb, ctgb, freq, ncontig, C.byref(pn),
                                                 C.byref(nl), C.byref(pc), C.byref(cl), nb, cb),
                 "self_adaptamer_merge")
        sb = 1 + 2 * (posb + ctgb)
        ns = _take(self.L, pn, nl.value).reshape(-1, sb)
        css = _take(self.L, pc, cl.value).reshape(-1, sb)
        return ns, css, nb, cb

    def reimport_sort(self, seeds: np.ndarray, posb: int, ctgb: int, comp: int, ncontig: int,
                      amxpos: int, dbyte: int):
        seeds = np.ascontiguousarray(seeds, dtype=np.uint8)
        swide = 2 * dbyte + ctgb + 2
        ns = seeds.shape[0]
        out = np.zeros((ns, swide), dtype=np.uint8)
        off = np.zeros(ncontig + 1, dtype=np.int64)
        self._ck(self.L.pga_reimport_sort(self.h, _ptr(seeds), seeds.size, posb, ctgb, comp, ncontig, amxpos,
                                          dbyte, _ptr(out), off), "reimport_sort")
        return out, off

    # ---- resident pipeline ---------------------------------------------------
    def index_build(self, want_entries: bool = True) -> int:
        n = C.c_int64()
        self._ck(self.L.pga_index_build(self.h, 1 if want_entries else 0, C.byref(n)), "index_build")
        self.nrec = n.value
        return n.value

    def index_records(self) -> np.ndarray:
        rs = self.record_sizing()[2]
        out = np.zeros((self.nrec, rs), dtype=np.uint8)
        self._ck(self.L.pga_index_copy_records(self.h, _ptr(out)), "index_copy_records")
        return out

    def index_entries(self):
        posb, ctgb, _ = self.record_sizing()
        ent = np.zeros((self.nrec, 9 + posb + ctgb), dtype=np.uint8)
        cum = np.zeros(1 << 24, dtype=np.int64)
        big = C.c_int64()
        self._ck(self.L.pga_index_copy_entries(self.h, _ptr(ent), cum.ctypes.data_as(vp), C.byref(big)),
                 "index_copy_entries")
        return ent, cum, big.value

    def merge(self, freq: int = 10):
        a, b = C.c_int64(), C.c_int64()
        self._ck(self.L.pga_merge(self.h, freq, C.byref(a), C.byref(b)), "merge")
        self.nseeds = [a.value, b.value]
        self._seeds_loaded = False
        return a.value, b.value

    def seeds(self, comp: int):
        posb, ctgb, _ = self.record_sizing()
        sb = 1 + 2 * (posb + ctgb)
        out = np.zeros((self.nseeds[comp], sb), dtype=np.uint8)
        buck = np.zeros(self.ncontig, dtype=np.int64)
        self._ck(self.L.pga_seeds_copy(self.h, comp, _ptr(out), buck.ctypes.data_as(vp)), "seeds_copy")
        return out, buck

    def seeds_load(self, comp: int, seeds: np.ndarray):
        """Unit comp's seeds in the reference's byte format (pga_seeds_load),
        in place of the merge's; the first load after a merge leaves the
        other unit empty until it is loaded too."""
        a = np.ascontiguousarray(seeds, dtype=np.uint8)
        buf = a if a.size else np.zeros(1, np.uint8)
        self._ck(self.L.pga_seeds_load(self.h, comp, _ptr(buf), int(a.size)), "seeds_load")
        posb, ctgb, _ = self.record_sizing()
        if not getattr(self, "_seeds_loaded", False):
            self.nseeds = [0, 0]
            self._seeds_loaded = True
        self.nseeds[comp] = a.size // (1 + 2 * (posb + ctgb))

    def diag_sort(self, comp: int):
        sw, n = C.c_int(), C.c_int64()
        self._ck(self.L.pga_diag_sort(self.h, comp, C.byref(sw), C.byref(n)), "diag_sort")
        return sw.value, n.value

    def diag_records(self, comp: int, swide: int, count: int):
        out = np.zeros((count, swide), dtype=np.uint8)
        off = np.zeros(self.ncontig + 1, dtype=np.int64)
        self._ck(self.L.pga_diag_copy(self.h, comp, _ptr(out), off.ctypes.data_as(vp)), "diag_copy")
        return out, off

    # ---- alignment -------------------------------------------------------------
    def set_freq(self, freq):
        f = np.ascontiguousarray(freq, dtype=np.float32)
        self._ck(self.L.pga_gdb_set_freq(self.h, f.ctypes.data_as(vp)), "gdb_set_freq")

    def align(self) -> int:
        n = C.c_int64()
        self._ck(self.L.pga_align(self.h, C.byref(n)), "align")
        self.nalign = n.value
        return n.value

    def align_times(self) -> dict:
        """Host wall-clock split of the last align() in ms."""
        a = (C.c_float * 4)()
        self._ck(self.L.pga_align_times(self.h, a), "align_times")
        return {"setup": a[0], "pairs": a[1], "self_pairs": a[2], "order": a[3]}

    def write_1aln(self, path, skeleton=None, db_name="", cwd=None, command="distributedpanga_b200", binary=True):
        """The last align()'s alignments as a .1aln file, in ONE's binary
        encoding as the reference writes it, or (binary=False) its ASCII one."""
        sk = skeleton or Skeleton.per_contig(self.cs.clen)
        names = sk.c_names()
        fn = self.L.pga_align_write_1aln_binary if binary else self.L.pga_align_write_1aln
        self._ck(fn(self.h, path.encode(), _PROG, _VERSION, command.encode(), db_name.encode(),
                    cwd.encode() if cwd else None, len(sk.names), names, sk.scaff_len.ctypes.data_as(vp),
                    sk.fctg.ctypes.data_as(vp), sk.sbeg.ctypes.data_as(vp)), "align_write_1aln")

    def local_alignment(self, requests):
        """Local_Alignment for each request row (a, b, comp, low, hgh, anti,
        lbord, hbord) on the loaded contigs.  Returns (paths (n, 7) int32:
        abpos aepos bbpos bepos diffs tlen status, trace offsets (n+1), trace
        uint16 values)."""
        req = np.ascontiguousarray(requests, dtype=np.int32).reshape(-1, 8)
        n = len(req)
        nt = C.c_int64()
        self._ck(self.L.pga_local_alignment(self.h, n, req.ctypes.data_as(vp) if n else None, C.byref(nt)),
                 "local_alignment")
        path = np.zeros((n, 7), dtype=np.int32)
        toff = np.zeros(n + 1, dtype=np.int64)
        tr = np.zeros(max(1, nt.value), dtype=np.uint16)
        self._ck(self.L.pga_local_alignment_copy(self.h, path.ctypes.data_as(vp), toff.ctypes.data_as(vp),
                                                 tr.ctypes.data_as(vp)), "local_alignment_copy")
        return path, toff, tr[: nt.value]

    def align_work(self) -> dict:
        """Wave steps, diagonal updates (cells), calls and warp tasks of the last align()."""
        a = np.zeros(4, dtype=np.int64)
        self._ck(self.L.pga_align_work(self.h, a.ctypes.data_as(vp)), "align_work")
        return {"waves": int(a[0]), "cells": int(a[1]), "calls": int(a[2]), "tasks": int(a[3])}

    def align_profile(self) -> dict:
        """Warp cycles of the last align(): inside Local_Alignment and in the
        pairs' finishing steps (summed over warps)."""
        a = np.zeros(2, dtype=np.int64)
        self._ck(self.L.pga_align_profile(self.h, a.ctypes.data_as(vp)), "align_profile")
        return {"local_alignment_cycles": int(a[0]), "finish_cycles": int(a[1])}

    def set_build(self, ctas_per_sm: int):
        """Which build of the alignment kernel runs (0 automatic, or 2 to 5 CTAs per SM)."""
        self._ck(self.L.pga_align_set_build(self.h, int(ctas_per_sm)), "align_set_build")

    def set_long_waves(self, waves: int) -> None:
        """Wave steps after which a call keeps its SM to itself (0 off, -1 automatic)."""
        self._ck(self.L.pga_align_set_long_waves(self.h, int(waves)), "align_set_long_waves")

    def set_digit_bits(self, bits: int) -> None:
        """Width of the index sort's first-level digit (0 automatic, 18..22)."""
        self._ck(self.L.pga_index_set_digit_bits(self.h, int(bits)), "index_set_digit_bits")

    def set_ranges(self, range_seeds: int) -> None:
        """Band-range size for large pairs (0 automatic, -1 never split)."""
        self._ck(self.L.pga_align_set_ranges(self.h, int(range_seeds)), "align_set_ranges")

    def alignments(self):
        """(records (n, 9) int32: aread abpos aepos bread bbpos bepos comp diffs tlen,
        trace offsets (n+1), trace bytes) in la_sort order."""
        n = self.nalign
        recs = np.zeros((n, 9), dtype=np.int32)
        toff = np.zeros(n + 1, dtype=np.int64)
        self._ck(self.L.pga_align_copy(self.h, recs.ctypes.data_as(vp), toff.ctypes.data_as(vp), None),
                 "align_copy")
        tr = np.zeros(max(1, int(toff[-1])), dtype=np.uint8)
        self._ck(self.L.pga_align_copy(self.h, None, None, tr.ctypes.data_as(vp)), "align_copy")
        return recs, toff, tr[: int(toff[-1])]

    def reuse_stats(self) -> dict:
        """The last alignment's use of a resident target's record of its own
        Local_Alignment calls (pga_align_reuse_stats): calls answered from
        it, of all calls made."""
        a = np.zeros(4, dtype=np.int64)
        self._ck(self.L.pga_align_reuse_stats(self.h, a.ctypes.data_as(vp)), "align_reuse_stats")
        why = {0: None, 1: "no record", 3: "scoring tables differ"}
        return {"used": bool(a[0]), "calls_from_record": int(a[1]), "calls": int(a[2]),
                "not_used": why.get(int(a[3]))}

    def align_stats(self) -> dict:
        a = np.zeros(8, dtype=np.int64)
        self._ck(self.L.pga_align_stats(self.h, a.ctypes.data_as(vp)), "align_stats")
        return {"pairs": int(a[0]), "self_pairs": int(a[1]), "calls": int(a[2]), "alignments": int(a[4]),
                "self_rounds": int(a[5]), "max_task_cycles": int(a[3]), "all_task_cycles": int(a[6]),
                "max_task_calls": int(a[7])}


class Target:
    """A resident target (pga_target): a FASTA text ingested and indexed on
    one device and kept there, read-only, for any number of contexts'
    requests (Device.serve_load).  With reuse, the target's own GDB is also
    aligned (FREQ = freq) and every Local_Alignment call it makes is kept: a
    request's call on two target contigs with the same inputs takes the kept
    result instead of being run (pga_target_create_reuse; same results)."""

    def __init__(self, text, nthr: int = 0, device: int = 0, reuse: bool = False, freq: int = 10):
        self.L = load_library()
        d = Device(device)
        try:
            d.gdb_ingest_fasta(text, nthr=nthr, tables=False)
            d.index_build(want_entries=False)
            h = vp()
            if reuse:
                d._ck(self.L.pga_target_create_reuse(d.h, freq, C.byref(h)), "target_create_reuse")
            else:
                d._ck(self.L.pga_target_create(d.h, C.byref(h)), "target_create")
        finally:
            d.close()
        self.reuse = reuse
        self.h = h
        self.device = device
        a = np.zeros(4, dtype=np.int64)
        self.L.pga_target_info(self.h, a.ctypes.data_as(vp))
        self.ncontig, self.bases, self.nrec, self.device_bytes = (int(x) for x in a)

    def close(self):
        if self.h:
            self.L.pga_target_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GdbTables:
    """A GDB as Create_GDB builds it (lib/GDB.h:28-70): the .bps image,
    contigs rows {clen, boff, sbeg, scaf}, scaffolds rows {fctg, ectg, slen,
    hoff}, the header block (names ended by NUL) and the base counts."""

    def __init__(self, bps, contigs, scaffolds, headers, count, maxctg):
        self.bps = bps
        self.contigs = contigs
        self.scaffolds = scaffolds
        self.headers = headers
        self.count = count
        self.maxctg = maxctg

    @property
    def seqtot(self) -> int:
        return int(self.count.sum())

    @property
    def freq(self) -> np.ndarray:
        """GDB.freq (lib/GDB.c:1083-1086)."""
        return (self.count / max(1, self.seqtot)).astype(np.float32)

    @property
    def names(self) -> list:
        return [self.headers[h:self.headers.index(b"\0", h)] for h in self.scaffolds[:, 3]]

    def skeleton(self) -> "Skeleton":
        fctg = np.append(self.scaffolds[:, 0], self.scaffolds[-1, 1] if len(self.scaffolds) else 0)
        return Skeleton(self.names, self.scaffolds[:, 2], fctg, self.contigs[:, 2])


class Skeleton:
    """The GDB skeleton of a .1aln file: scaffold names and lengths, and
    where each contig sits (contigs of scaffold s are fctg[s]..fctg[s+1]-1,
    contig c at sbeg[c] within its scaffold).  One contig per scaffold when
    built from plain contig lengths."""

    def __init__(self, names, scaff_len, fctg, sbeg):
        self.names = [n.encode() if isinstance(n, str) else bytes(n) for n in names]
        self.scaff_len = np.ascontiguousarray(scaff_len, dtype=np.int64)
        self.fctg = np.ascontiguousarray(fctg, dtype=np.int32)
        self.sbeg = np.ascontiguousarray(sbeg, dtype=np.int64)

    @classmethod
    def per_contig(cls, clen, names=None):
        clen = np.asarray(clen, dtype=np.int64)
        n = len(clen)
        names = names if names is not None else ["ctg%d" % i for i in range(n)]
        return cls(names, clen, np.arange(n + 1, dtype=np.int32), np.zeros(n, dtype=np.int64))

    def c_names(self):
        arr = (C.c_char_p * max(1, len(self.names)))(*self.names)
        return arr


_PROG = b"distributedpanga_b200"
_VERSION = b"0.1"


def write_1aln(path, recs, toff, trace, contig_len, skeleton=None, db_name="", cwd=None,
               command="distributedpanga_b200", tspace=100, binary=True):
    """Writes alignments (as Device.alignments() returns them) as a .1aln file
    (la_merge's output, src/fastga_pipeline.c:1616-1656), in ONE's binary
    encoding as the reference writes it, or (binary=False) its ASCII one."""
    L = load_library()
    contig_len = np.ascontiguousarray(contig_len, dtype=np.int64)
    sk = skeleton or Skeleton.per_contig(contig_len)
    recs = np.ascontiguousarray(recs, dtype=np.int32)
    toff = np.ascontiguousarray(toff, dtype=np.int64)
    trace = np.ascontiguousarray(trace, dtype=np.uint8)
    if trace.size == 0:
        trace = np.zeros(1, dtype=np.uint8)
    names = sk.c_names()
    fn = L.pga_write_1aln_binary if binary else L.pga_write_1aln
    rc = fn(path.encode(), _PROG, _VERSION, command.encode(), db_name.encode(), cwd.encode() if cwd else None,
            int(tspace), len(sk.names), names, sk.scaff_len.ctypes.data_as(vp), sk.fctg.ctypes.data_as(vp),
            sk.sbeg.ctypes.data_as(vp), contig_len.ctypes.data_as(vp), int(len(recs)), recs.ctypes.data_as(vp),
            toff.ctypes.data_as(vp), trace.ctypes.data_as(vp))
    if rc != 0:
        raise PgaError("write_1aln(%s): status %d" % (path, rc))


def read_gix(stem):
    """A GIX on disk (<stem>.gix and the .ktab parts beside it, from GIXmake
    or Device.index_write_gix) as the k-mer table view: {"kmer", "parts",
    "post_bytes", "cont_bytes", "freq", "order", "cum", "largest",
    "entries"}, contigs numbered as in the GDB (pga_read_gix)."""
    L = load_library()
    hdr = np.zeros(6, dtype=np.int32)
    largest, n = C.c_int64(), C.c_int64()
    rc = L.pga_read_gix(stem.encode(), hdr.ctypes.data_as(vp), None, 0, None, C.byref(largest), C.byref(n), None, 0)
    if rc != 0:
        raise PgaError("read_gix(%s): status %d" % (stem, rc))
    eb = 9 + int(hdr[2]) + int(hdr[3])
    order = np.zeros(max(1, int(hdr[5])), dtype=np.int32)
    cum = np.zeros(1 << 24, dtype=np.int64)
    ent = np.zeros((max(1, n.value), eb), dtype=np.uint8)
    rc = L.pga_read_gix(stem.encode(), hdr.ctypes.data_as(vp), order.ctypes.data_as(vp), len(order),
                        cum.ctypes.data_as(vp), C.byref(largest), C.byref(n), ent.ctypes.data_as(vp), n.value)
    if rc != 0:
        raise PgaError("read_gix(%s): status %d" % (stem, rc))
    return {"kmer": int(hdr[0]), "parts": int(hdr[1]), "post_bytes": int(hdr[2]), "cont_bytes": int(hdr[3]),
            "freq": int(hdr[4]), "order": order[:int(hdr[5])], "cum": cum, "largest": largest.value,
            "entries": ent[:n.value]}


def alignment_lines(recs, toff, tr):
    """The .1aln record stream as text, one alignment per line:
    aread abpos aepos bread bbpos bepos comp diffs ; T b-deltas ; X diffs."""
    out = []
    for i, r in enumerate(recs):
        t = tr[toff[i]:toff[i + 1]]
        out.append("%d %d %d %d %d %d %d %d ; %s ; %s" % (r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7],
                                                          " ".join(map(str, t[1::2].tolist())),
                                                          " ".join(map(str, t[0::2].tolist()))))
    return out
