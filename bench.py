"""Benchmark of the GPU alignment path.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload full|chromset|pangenome]

Default workload: two 1 Gbp genomes in one GDB (the 2 x 1 Gbp configuration,
`full`), with the 2 x 100 Mbp chromosome-set configuration (`chromset`)
measured after it as the line's `secondary` object.

One step = one pass of the whole alignment path over the contig set, inputs
resident in HBM: closed-syncmer extraction -> 24-bit-prefix bucket sort ->
semantic LCPs -> adaptamer merge -> seed reimport + diagonal sort of the N
and C units -> chaining and Local_Alignment of every contig pair
(FastGA-order self pairs) -> the alignment records in la_sort order, left
in HBM.  The k-mer table entries in the reference's byte layout are written
only with --entries (nothing on the path reads them).

value  = input bases (both genomes, Mbp) per second of device time, max over
         ranks
e2e    = the same through the C ABI with host buffers: every e2e step uploads
         the .bps image and contig table from pinned host memory, runs the
         path and reads the alignment records and traces back to the host
         (--e2e-steps steps after one warm-up)
roofline = the index build (extract + sort + LCP [+ entries]), whose
         algorithmic bytes are ceil(G/4) + 5*N*R [+ N*E] + 2^27
bit_exact = the secondary (2 x 100 Mbp) workload's index, seeds, sorted
         diagonal panels and .1aln record stream against digests of the
         reference's own pipeline on the same seeded input
         (tests/golden/chromset_full.json), checked outside the timed region
cpu_baseline = the reference pipeline compiled from source (oracle/_ref), or
         the oracle's C restatement when that is absent, on a bounded sample
         of the same generator; the secondary object's cpu_baseline is the
         reference on the whole 2 x 100 Mbp input (the same bytes)
--impl reference = the reference pipeline (oracle/_ref) on every host core:
         one concurrent world-1 run per core on a sample, the aggregate rate
         (its driver has one alignment thread and gets its parallelism from
         MPI ranks, which this host does not have)
served_form = a resident 1 Gbp target (with the record of its own
         Local_Alignment calls) against a Poisson stream of 12 query
         assemblies, beside the plain form on the same requests; every served
         result is compared with the plain one

With N > 1 every rank runs an independent replica (the path has no exchange
step on one node's workload): weak scaling, no collective in the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "aligned Mbp/s per B200 (input bases of both genomes / end-to-end seconds, plain method)"
UNIT = "Mbp/s"
WORKLOADS = {
    "chromset": "chromset: 2 x 100 Mbp, 40% GC, log-normal contigs (median 2 Mbp, sigma 1), 10% repeats; k=40, FREQ=10",
    "full": "full: 2 x 1 Gbp, uniform ACGT, contigs U[50, 500] kbp, 40% interspersed repeats, 3% tandem arrays, "
            "B = A at 2% substitutions + 0.5% indels + 20 inversions; k=40, FREQ=10",
    "pangenome": "pangenome: a 50 Mbp reference + 16 haplotypes (0.1-1% substitutions, a tenth as indels, "
                 "10 inversions + 5 translocations each), log-normal contigs 10 kbp-5 Mbp, all in one GDB; "
                 "k=40, FREQ=10 (the reference driver's cutoff)",
}
WL = {"name": "full"}  # the workload being measured
FREQ = {}              # frequency cutoff per workload (10, the reference driver's, unless listed)
# golden digests of the reference's pipeline for a workload at a scale
GOLDEN = {("chromset", 1.0): "chromset_full", ("full", 0.01): "full_s001", ("pangenome", 0.02): "pangenome_s002"}
# CPU samples of each generator: the reference arm's per-step sample and the
# cpu_baseline sample (about 10 s and 20 s of the reference's pipeline here)
REF_SCALE = {"full": 0.004, "chromset": 0.05, "pangenome": 0.01}
CPU_SCALE = {"full": 0.01, "chromset": 0.1, "pangenome": 0.02}


def freq_cutoff() -> int:
    return FREQ.get(WL["name"], 10)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.p = None
        self.out = ""

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            self.out += line

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().split("\n"):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def make_contigs(scale: float, name: str | None = None):
    from distributedpanga_b200 import gdb, synth
    name = name or WL["name"]
    cache = os.path.join(tempfile.gettempdir(), "pga_%s_%g.npz" % (name, scale))
    if os.path.exists(cache):
        z = np.load(cache)
        return gdb.ContigSet(bps=z["bps"], clen=z["clen"], boff=z["boff"], freq=z["freq"]), None
    contigs = synth.make(name, scale=scale)
    cs = gdb.from_contigs(contigs)
    try:  # written whole, then renamed: ranks of one run may build it at once
        tmp = "%s.%d.tmp.npz" % (cache[:-4], os.getpid())
        np.savez(tmp, bps=cs.bps, clen=cs.clen, boff=cs.boff, freq=cs.freq)
        os.replace(tmp, cache)
    except OSError:
        pass
    return cs, contigs


def index_bytes(cs, nrec: int, entries: bool = True) -> float:
    from distributedpanga_b200 import gdb
    posb, ctgb, rsize = gdb.record_sizing(cs)
    ebytes = rsize - 3 if entries else 0
    return (cs.seqtot + 3) // 4 + 5.0 * nrec * rsize + nrec * ebytes + (1 << 27)


# ---- reference / oracle CPU timing -------------------------------------------

class ReferenceSample:
    """The reference pipeline (oracle/_ref) on a sample of a workload's
    generator: the GDB and its .gix (GIXmake from source, whose contig order
    src/fastga_order.c reads; its own text dump off) are built once,
    untimed; each run() times one pga-mpi-merge and returns the seconds of
    its own stage timers."""

    def __init__(self, scale: float, name: str | None = None):
        from distributedpanga_b200 import gdb, synth
        from oracle import binding as orc
        self.name = name or WL["name"]
        self.tmp = tempfile.TemporaryDirectory()
        contigs = synth.make(self.name, scale=scale)
        self.mbp = gdb.from_contigs(contigs).seqtot / 1e6
        fa = os.path.join(self.tmp.name, "s.fa")
        self.stem = os.path.join(self.tmp.name, "s")
        synth.write_fasta(fa, contigs)
        orc.ref_make_gdb(fa, self.stem)
        env = dict(os.environ)
        env["GIXMAKE_DUMP_PATH"] = os.devnull
        with open(os.path.join(self.tmp.name, "gix.log"), "w") as log:
            # untimed set-up, one thread: on a loaded host GIXmake's threaded
            # build is slower here and now and then writes an entry's LCP against
            # the wrong predecessor (the driver reads only the .gix header and its
            # contig order, src/fastga_order_core.c:11-48)
            subprocess.run([os.path.join(orc.REF_DIR, "GIXmake_dump"), "-T1", self.stem + ".1gdb"], check=True,
                           stdout=log, stderr=subprocess.STDOUT, cwd=self.tmp.name, env=env)

    def run(self, whole: bool = True) -> float:
        from oracle import binding as orc
        env = dict(os.environ)
        env["PATH"] = orc.REF_DIR + os.pathsep + env.get("PATH", "")
        env.setdefault("PGA_SCRATCH_DIR", tempfile.gettempdir())
        logp = os.path.join(self.tmp.name, "merge.log")
        with open(logp, "w") as log:
            subprocess.run([os.path.join(orc.REF_DIR, "pga-mpi-merge"), self.stem], check=True, stdout=log,
                           stderr=subprocess.STDOUT, cwd=self.tmp.name, env=env)
        text = open(logp).read()
        if whole:
            # the driver's own stage timers: extract, sort, merge, alignments
            # (src/pga-mpi-merge.c:669-688); alignments includes ALNtoPAF, here a copy
            tot = re.search(r"TOTAL\s+([0-9.]+)s", text)
            return float(tot.group(1))
        o1 = dict(re.findall(r"(\w+)=([0-9.]+)", text.split("[o1-0]")[1].split("\n")[0]))
        pr = dict(re.findall(r"(\w+)=([0-9.]+)", text.split("[pr1]")[1].split("\n")[0]))
        return (float(o1["extract_s"]) + float(o1["sort_stage_s"]) + float(pr["adapter_s"]) +
                float(pr["merge_core_s"]) + float(pr["reimport_n_s"]) + float(pr["reimport_c_s"]) +
                float(pr["sort_n_s"]) + float(pr["sort_c_s"]))


    def run_many(self, k: int) -> float:
        """k concurrent runs of the reference's pipeline on the sample, each
        world 1 in its own directory; returns the slowest run's TOTAL stage
        time.  The reference gets its parallelism from MPI ranks and its
        driver runs one alignment thread (NTHREADS, src/pga-mpi-merge.c:55);
        with no MPI on the host, k ranks that exchange nothing are the most
        of the host it could use (an upper bound on its k-rank rate)."""
        from oracle import binding as orc
        env = dict(os.environ)
        env["PATH"] = orc.REF_DIR + os.pathsep + env.get("PATH", "")
        env.setdefault("PGA_SCRATCH_DIR", tempfile.gettempdir())
        procs, logs = [], []
        for i in range(k):
            d = os.path.join(self.tmp.name, "r%d" % i)
            os.makedirs(d, exist_ok=True)
            logp = os.path.join(d, "merge.log")
            logs.append(logp)
            with open(logp, "w") as log:
                procs.append(subprocess.Popen([os.path.join(orc.REF_DIR, "pga-mpi-merge"), self.stem], stdout=log,
                                              stderr=subprocess.STDOUT, cwd=d, env=env))
        bad = [p.wait() for p in procs]
        if any(bad):
            raise RuntimeError("reference run failed: exit codes %s" % bad)
        tot = [float(re.search(r"TOTAL\s+([0-9.]+)s", open(l).read()).group(1)) for l in logs]
        return max(tot)


def port_sample(scale: float, name: str | None = None):
    """The oracle's C restatement on a sample; returns (Mbp, seconds)."""
    from distributedpanga_b200 import gdb, synth
    from oracle import binding as orc
    cs = gdb.from_contigs(synth.make(name or WL["name"], scale=scale))
    posb, ctgb, _ = gdb.record_sizing(cs)
    dbyte, _ = gdb.diag_sizing(cs, ctgb)
    t0 = time.time()
    srt = orc.sort_records(orc.extract(cs, posb, ctgb))
    ent, cum, _ = orc.build_adapter(srt, posb, ctgb)
    ns, css, _, _ = orc.merge(ent, cum, posb, ctgb, freq_cutoff(), cs.ncontig)
    orc.reimport_sort(ns, posb, ctgb, 0, cs.ncontig, cs.maxctg, dbyte)
    orc.reimport_sort(css, posb, ctgb, 1, cs.ncontig, cs.maxctg, dbyte)
    return cs.seqtot / 1e6, time.time() - t0


def cpu_baseline(sample_scale: float, name: str | None = None) -> dict:
    """The reference's whole pipeline (its TOTAL stage time) on a sample of
    the workload's generator, once; host cores stated."""
    from oracle import binding as orc
    name = name or WL["name"]
    cores_total = os.cpu_count()
    if orc.ref_available():
        r = ReferenceSample(sample_scale, name)
        sec = r.run()
        mbp = r.mbp
        return {"value": mbp / sec, "unit": UNIT, "cores": 4, "kind": "reference",
                "sample": name + " generator at scale %g (%.1f Mbp), reference pga-mpi-merge world 1 "
                          "(oracle/_ref), whole path (its TOTAL stage time: extract, sort, merge, alignments); "
                          "msd_sort uses 4 threads, the rest 1; host has %d cores" % (sample_scale, mbp, cores_total),
                "seconds": sec}
    orc.build()
    mbp, sec = port_sample(sample_scale, name)
    return {"value": mbp / sec, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": name + " generator at scale %g (%.1f Mbp), oracle C restatement (extract to diagonal sort), "
                      "1 thread; host has %d cores" % (sample_scale, mbp, cores_total), "seconds": sec}


# ---- GDB ingest ------------------------------------------------------------------

def fasta_text(cs) -> bytes:
    """The workload as the FASTA the reference's GDB is made from: one scaffold
    ctg<i> per contig, 80 bases a line (synth.write_fasta's layout)."""
    letters = np.frombuffer(b"ACGT", np.uint8)
    parts = []
    for i in range(cs.ncontig):
        s = letters[cs.contig(i)]
        full = len(s) // 80
        rows = np.empty((full, 81), np.uint8)
        rows[:, :80] = s[:full * 80].reshape(full, 80)
        rows[:, 80] = 10
        tail = s[full * 80:].tobytes()
        parts.append(b">ctg%d\n" % i + rows.tobytes() + (tail + b"\n" if tail else b""))
    return b"".join(parts)


def ingest_cpu_baseline(text: bytes, sample_bytes: int) -> dict:
    """Create_GDB on the host for the first scaffolds of `text` (about
    sample_bytes): the reference's own reader (oracle/_ref/fa2gdb) when built,
    else the oracle's restatement."""
    from oracle import binding as orc
    cut = text.find(b"\n>", sample_bytes)
    sample = text if cut < 0 else text[:cut + 1]
    fa2gdb = os.path.join(orc.REF_DIR, "fa2gdb")
    if os.path.exists(fa2gdb):
        with tempfile.TemporaryDirectory() as d:
            fa = os.path.join(d, "s.fa")
            with open(fa, "wb") as f:
                f.write(sample)
            best = None
            for _ in range(3):
                t0 = time.perf_counter()
                subprocess.run([fa2gdb, fa, os.path.join(d, "s.1gdb")], check=True, capture_output=True)
                sec = time.perf_counter() - t0
                best = sec if best is None else min(best, sec)
        return {"value": len(sample) / best / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
                "sample": "first %.1f MB of the workload's FASTA, reference Create_GDB + Write_GDB "
                          "(oracle/_ref/fa2gdb, file in page cache, best of 3)" % (len(sample) / 1e6),
                "seconds": best}
    orc.build()
    t0 = time.perf_counter()
    orc.fasta_gdb(sample, 0)
    sec = time.perf_counter() - t0
    return {"value": len(sample) / sec / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": "first %.1f MB of the workload's FASTA, oracle restatement of Create_GDB's reader"
                      % (len(sample) / 1e6), "seconds": sec}


def run_ingest(dev, cs, args, stream, peak: float, peak_kind: str, cpu: bool) -> dict:
    """pga_gdb_ingest_fasta on the workload's FASTA from pinned host memory:
    upload + parse timed per call with CUDA events; the GDB it builds must be
    the one the alignment path was measured on."""
    import torch
    text = fasta_text(cs)
    n = len(text)
    pinned = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = np.frombuffer(text, np.uint8)
    ptr = pinned.data_ptr()
    calls, parse, upload = [], [], []
    sizes = None
    for it in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        sizes = dev.gdb_ingest_fasta(ptr, 0, nbytes=n, tables=False)
        t1.record(stream)
        torch.cuda.synchronize()
        if it >= args.warmup:
            calls.append(t0.elapsed_time(t1))
            tm = dev.gdb_ingest_times()
            parse.append(tm["parse_ms"])
            upload.append(tm["upload_ms"])
    t = dev.gdb_tables(sizes)
    same = bool(np.array_equal(t.bps, cs.bps) and np.array_equal(t.contigs[:, 0], cs.clen)
                and np.array_equal(t.contigs[:, 1], cs.boff))
    parse_ms, call_ms = statistics.median(parse), statistics.median(calls)
    alg = n + int(sizes[2])
    out = {"input_bytes": n, "scaffolds": int(sizes[0]), "contigs": int(sizes[1]), "bps_bytes": int(sizes[2]),
           "identical_to_benchmarked_gdb": same,
           "call_ms": call_ms, "upload_ms": statistics.median(upload), "parse_ms": parse_ms,
           "e2e_gbs": n / (call_ms / 1000.0) / 1e9, "parse_gbs": n / (parse_ms / 1000.0) / 1e9,
           "roofline": {"bound": "hbm", "kernel": "FASTA parse (header scan, sequence compaction, N runs, "
                                                  "contig layout, 2-bit pack)",
                        "achieved": alg / (parse_ms / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / (parse_ms / 1000.0) / 1e9 / peak, "peak_source": peak_kind,
                        "algorithmic_bytes": alg, "note": "text read once + image written once"}}
    if cpu:
        try:
            out["cpu_baseline"] = ingest_cpu_baseline(text, 24 << 20)
        except Exception as e:
            out["cpu_baseline"] = {"value": None, "sample": "failed: %s" % e}
    return out


def run_profile_stage(args) -> None:
    """--profile-stage: one stage alone (index build, GDB ingest, served load,
    alignment launch or diagonal sorts), warmup + steps times on one GPU,
    printing each call's device times (a small program for ncu captures of
    one stage's kernels)."""
    from distributedpanga_b200 import pipeline
    if args.profile_stage == "serve":
        # the served load alone: a target at --serve-scale, then queries
        # ingested and merged into its index (k_union_rank), one per call
        from distributedpanga_b200 import synth
        sc = args.serve_scale
        contigs = synth.make_target(scale=sc)
        target = pipeline.Target(synth.fasta_bytes(contigs, "t"))
        stream = synth.query_stream(contigs, args.warmup + args.steps, 0.0, int(1_000_000 * sc),
                                    int(200_000_000 * sc), seed=31, median=2_000_000 * max(sc, 0.05))
        dev = pipeline.Device(0)
        for k, (_, q) in enumerate(stream):
            t = time.perf_counter()
            sizes = dev.serve_load(target, synth.fasta_bytes(q, "q%d_" % k))
            print(json.dumps({"stage": "serve_load", "target_records": target.nrec, "records": dev.nrec,
                              "query_bases": int(sizes[5]) - target.bases,
                              "ms": round(1000 * (time.perf_counter() - t), 3)}), flush=True)
        dev.close()
        target.close()
        return
    cs, _ = make_contigs(args.scale)
    dev = pipeline.Device(0)
    if args.profile_stage == "align":
        # the alignment launch alone: the index, merge and diagonal sorts once,
        # then warmup + steps alignments with the chosen kernel build
        dev.gdb_load(cs)
        dev.index_build(want_entries=False)
        dev.merge(freq_cutoff())
        dev.diag_sort(0)
        dev.diag_sort(1)
        dev.set_build(args.align_build)
        for _ in range(args.warmup + args.steps):
            n = dev.align()
            print(json.dumps({"stage": "align", "alignments": n, "work": dev.align_work(),
                              "times_ms": dev.align_times()}), flush=True)
        dev.close()
        return
    if args.profile_stage == "diag":
        # the diagonal sorts alone: the index once, then warmup + steps of
        # merge (the sort consumes the seeds) + both units' sorts
        dev.gdb_load(cs)
        dev.index_build(want_entries=False)
        dev.enable_timing(True)
        for _ in range(args.warmup + args.steps):
            dev.merge(freq_cutoff())
            dev.diag_sort(0)
            dev.diag_sort(1)
            st = dev.stage_times()
            print(json.dumps({"stage": "diag", "seeds": dev.nseeds,
                              "ms": {k: round(st[k], 3) for k in ("merge", "diag_sort_n", "diag_sort_c")}}),
                  flush=True)
        dev.close()
        return
    if args.profile_stage == "index":
        dev.gdb_load(cs)
        if args.digit_bits:
            dev.set_digit_bits(args.digit_bits)
        dev.enable_timing(True)
        for _ in range(args.warmup + args.steps):
            n = dev.index_build(want_entries=args.entries)
            st = dev.stage_times()
            print(json.dumps({"stage": "index", "records": n,
                              "ms": {k: st[k] for k in ("extract_hist", "prefix_scan", "extract_scatter",
                                                        "bucket_sort", "lcp", "entries_prefix_table")}}),
                  flush=True)
    else:
        text = fasta_text(cs)
        for _ in range(args.warmup + args.steps):
            sizes = dev.gdb_ingest_fasta(text, 0, tables=False)
            print(json.dumps({"stage": "ingest", "bytes": len(text), "sizes": [int(x) for x in sizes],
                              "ms": dev.gdb_ingest_times()}), flush=True)
    dev.close()


def reference_runs() -> int:
    """Concurrent reference runs per step: one per usable host core, at most
    one per GiB of available memory (a run on the sample peaks near 0.2 GB)
    and at most 256."""
    cores = len(os.sched_getaffinity(0))
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError):
        avail = 1 << 40
    return max(1, min(cores, 256, avail >> 30))


def run_reference(args, rank: int) -> None:
    """The reference arm: the reference's own pipeline on all the host's
    cores, each step one concurrent world-1 run per core (reference_runs) on a
    sample of the workload's generator (REF_SCALE, or --ref-scale), the
    aggregate rate over the slowest run; rank 0 alone."""
    if rank != 0:
        return
    from oracle import binding as orc
    vals = []
    detail = None
    ref = ReferenceSample(args.ref_scale) if orc.ref_available() else None
    nrun = reference_runs()
    for it in range(args.warmup + args.steps):
        if ref is not None:
            mbp, sec = ref.mbp * nrun, ref.run_many(nrun)
            kind, cores = "reference", nrun
        else:
            orc.build()
            mbp, sec = port_sample(args.ref_scale)
            kind, cores = "port", 1
        if it >= args.warmup:
            vals.append(mbp / sec)
        detail = (mbp, kind, cores)
    v = statistics.median(vals)
    mbp, kind, cores = detail
    if kind == "reference":
        sample = (WL["name"] + " generator at scale %g (%.1f Mbp) per run, %d concurrent world-1 runs of the "
                  "reference pipeline per step (one per host core; its driver has one alignment thread and no MPI "
                  "is here), aggregate Mbp / the slowest run's TOTAL stage time"
                  % (args.ref_scale, mbp / cores, cores))
    else:
        sample = WL["name"] + " generator at scale %g (%.1f Mbp) per step" % (args.ref_scale, mbp)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mbp / v * 1000.0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOADS[WL["name"]], "sample_scale": args.ref_scale, "sample": sample},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    emit(rank, line)


# ---- ranks ---------------------------------------------------------------------------

def barrier(world: int) -> None:
    if world > 1:
        import torch
        torch.distributed.barrier()


def max_over_ranks(vals, world: int, device: str):
    """Element-wise maximum of `vals` over all ranks (the slowest rank's times)."""
    if world <= 1:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def emit(rank: int, line: dict) -> None:
    """Rank 0 prints the one JSON line."""
    if rank == 0:
        print(json.dumps(line), flush=True)


def align_roofline(work: dict, align_ms: float) -> dict:
    """The aligner is integer-issue bound: its work in cells (one diagonal
    updated in one wave step) per second, with the SM issue utilisation of
    k_align_pairs from the committed ncu summary when there is one (a capture
    on another, smaller workload: its source is stated)."""
    out = {"bound": "issue", "unit": "cells/s", "cells": work["cells"], "waves": work["waves"],
           "calls": work["calls"], "warp_tasks": work["tasks"],
           "achieved": work["cells"] / (align_ms / 1000.0) if align_ms > 0 else None,
           "issue_util": None, "issue_util_source": None}
    try:
        with open(os.path.join(ROOT, "profiles", "k_align_pairs_issue.json")) as f:
            prof = json.load(f)
        out["issue_util"] = prof.get("sm_issue_active_pct_of_active_cycles")
        out["issue_util_source"] = prof.get("source", "profiles/k_align_pairs_issue.json")
    except Exception:
        pass
    return out


def index_traffic(name: str, scale: float, nrec: int):
    """DRAM bytes per index build from a committed ncu capture of the index
    build on this workload's generator (profiles/traffic.json), scaled by the
    record count when the capture ran on a smaller case; with its source."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tr = json.load(f)
    except Exception:
        return None, None
    cap = tr.get("index_build", {}).get(name)
    if not cap:
        return None, None
    per_rec = cap["dram_bytes"] / cap["records"]
    src = "ncu capture of the index build on %s (%d records, %s), scaled by records" % (
        cap["case"], cap["records"], cap["file"])
    return per_rec * nrec, src


def golden_check(dev, name: str, scale: float) -> dict:
    """Every stage of one more pass on the loaded GDB against the golden
    digests of the reference's pipeline for this workload and scale (index,
    N and C seeds, sorted diagonal panels, .1aln record stream); outside the
    timed region.  {"bit_exact": true|false|null, ...}."""
    key = GOLDEN.get((name, scale))
    path = os.path.join(ROOT, "tests", "golden", "%s.json" % key) if key else None
    if not path or not os.path.exists(path):
        return {"bit_exact": None, "reason": "no reference digests for %s at scale %g" % (name, scale)}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import helpers as H
    from distributedpanga_b200.pipeline import alignment_lines
    with open(path) as f:
        dig = json.load(f)
    stage = "index"
    try:
        dev.index_build(want_entries=False)
        rec = dev.index_records()
        H.check_index_large(rec, dig)
        del rec
        stage = "seeds"
        dev.merge(dig["freq_cutoff"])
        ns, nb = dev.seeds(0)
        css, cb = dev.seeds(1)
        H.check_seeds_large(ns, css, nb, cb, dig)
        del ns, css
        for comp, u in ((0, "N"), (1, "C")):
            stage = "diag_" + u
            sw, cnt = dev.diag_sort(comp)
            arr, off = dev.diag_records(comp, sw, cnt)
            H.check_diag_large(arr, off, u, dig)
            del arr
        stage = "aln"
        dev.align()
        lines = [" ".join(x.split()) for x in alignment_lines(*dev.alignments())]
        H.check_lines(lines, dig["aln"])
    except AssertionError as e:
        return {"bit_exact": False, "first_difference": stage, "detail": str(e)[:200], "golden": key + ".json"}
    return {"bit_exact": True, "golden": key + ".json", "stages": "index, N/C seeds, N/C diagonal panels, .1aln",
            "alignments": dig["aln"]["count"]}


def measure(args, name: str, scale: float, steps: int, warmup: int, e2e_steps: int, rank: int, world: int,
            local_rank: int, check: bool) -> dict:
    """One workload on this rank's GPU: `warmup` untimed steps, `steps` timed
    steps (CUDA events on the launching stream, max over ranks), one more
    step with per-stage times, `e2e_steps` end-to-end steps through the C ABI
    from pinned host memory, and (check) the golden comparison."""
    import torch
    from distributedpanga_b200 import gdb, pipeline
    WL["name"] = name
    cs, _ = make_contigs(scale, name)
    posb, ctgb, rsize = gdb.record_sizing(cs)
    dev = pipeline.Device(local_rank)
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    dev.gdb_load(cs)
    tuned = None
    if args.autotune:
        # untimed: pick the launch parameters on this workload, then run with them
        from distributedpanga_b200 import autotune
        tu = autotune.Tuner(dev, repeats=2)
        cfg = tu.tune()
        autotune.apply(dev, cfg)
        tuned = {"chosen": cfg, "median_s": {k: {str(c): round(statistics.median(v), 4) for c, v in t.items()}
                                             for k, t in tu.times.items()}}

    def step():
        dev.index_build(want_entries=args.entries)
        dev.merge(freq_cutoff())
        dev.diag_sort(0)
        dev.diag_sort(1)
        dev.align()

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local_rank)
    clocks.start()
    l0 = dev.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = ev0.elapsed_time(ev1) / steps
    launches = (dev.launches() - l0) // steps
    clk = clocks.stop()
    nrec = dev.nrec
    nseeds = dev.nseeds

    # stage times of one more step
    dev.enable_timing(True)
    step()
    st = dev.stage_times()
    alloc = dev.alloc_times()
    dev.enable_timing(False)
    astats = dev.align_stats()
    atimes = dev.align_times()
    awork = dev.align_work()
    aprof = dev.align_profile()
    recs, toff, tr = dev.alignments()
    aligned_bases = int((recs[:, 2] - recs[:, 1]).sum()) if len(recs) else 0

    # end to end through the C ABI with host buffers: upload the GDB (its
    # .bps image from pinned host memory), run the path, read the alignments
    # back
    swide = None
    h2d = int(cs.bps.size + 16 * cs.ncontig)
    d2h = 0
    e2e_ms = []
    pinned = torch.empty(max(1, cs.bps.size), dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[: cs.bps.size] = cs.bps
    pcs = gdb.ContigSet(bps=pinned.numpy()[: cs.bps.size], clen=cs.clen, boff=cs.boff, freq=cs.freq)
    for it in range(1 + e2e_steps):
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        dev.gdb_load(pcs)
        dev.index_build(want_entries=args.entries)
        dev.merge(freq_cutoff())
        swide, _ = dev.diag_sort(0)
        dev.diag_sort(1)
        dev.align()
        r2, o2, t2 = dev.alignments()
        d2h = r2.nbytes + o2.nbytes + t2.nbytes
        t1.record(stream)
        torch.cuda.synchronize()
        if it >= 1:
            e2e_ms.append(t0.elapsed_time(t1))
    e2e_ms_step = statistics.median(e2e_ms)

    ms, e2e_ms_step = max_over_ranks([ms, e2e_ms_step], world, "cuda")
    mbp = cs.seqtot / 1e6
    value = world * mbp / (ms / 1000.0)
    e2e = world * mbp / (e2e_ms_step / 1000.0)

    out = {"value": value, "ms_per_step": ms, "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                                                      "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
           "gpu_launches": int(launches), "clocks": clk, "autotune": tuned, "cs": cs, "dev": dev}
    if rank != 0:
        dev.close()
        return out
    peak, peak_kind = peaks()
    idx_ms = sum(st[k] for k in ("extract_hist", "prefix_scan", "extract_scatter", "bucket_sort", "lcp",
                                 "entries_prefix_table"))
    ab = index_bytes(cs, nrec, args.entries)
    achieved = ab / (idx_ms / 1000.0) / 1e9
    traffic, traffic_src = index_traffic(name, scale, nrec)
    out.update({
        "config": {"workload": WORKLOADS[name], "scale": scale, "input_bases": cs.seqtot, "contigs": cs.ncontig,
                   "records": nrec, "seeds_n": nseeds[0], "seeds_c": nseeds[1],
                   "pairs": astats["pairs"], "self_pairs": astats["self_pairs"],
                   "local_alignment_calls": astats["calls"], "alignments": astats["alignments"],
                   "longest_warp_task_ms_at_max_clock": astats["max_task_cycles"] / 1965e3,
                   "longest_warp_task_calls": astats["max_task_calls"],
                   "all_tasks_warp_s_at_max_clock": astats["all_task_cycles"] / 1965e6,
                   "local_alignment_warp_s_at_max_clock": aprof["local_alignment_cycles"] / 1965e6,
                   "finish_warp_s_at_max_clock": aprof["finish_cycles"] / 1965e6,
                   "aligned_bases": aligned_bases, "record_bytes": rsize, "swide": swide,
                   "entries_written": bool(args.entries),
                   "l2": "inputs larger than L2 (records %.1f GB)" % (nrec * 16 / 1e9),
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "stage_ms": st,
        "alloc_ms": {k: round(v, 2) if isinstance(v, float) else v for k, v in alloc.items()},
        "align_ms": atimes,
        "align_roofline": align_roofline(awork, st["align"]),
        "roofline": {"bound": "hbm", "kernel": "index build (k_extract hist+scatter, prefix scan, bucket sort, "
                                               "k_lcp%s, k_prefix_table)" % (", k_entries" if args.entries else ""),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": traffic, "traffic_source": traffic_src,
                     "algorithmic_bytes": ab, "ms": idx_ms},
    })
    if check:
        out["golden"] = golden_check(dev, name, scale)
    return out


def run_ours(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    torch.cuda.set_device(local_rank)
    name = args.workload
    m = measure(args, name, args.scale, args.steps, args.warmup, min(args.steps, args.e2e_steps), rank, world,
                local_rank, check=world == 1 and not args.no_check)
    if rank != 0:
        return
    dev, cs = m.pop("dev"), m.pop("cs")
    peak, peak_kind = peaks()
    ingest = None
    if not args.no_ingest:
        stream = torch.cuda.current_stream()
        ingest = run_ingest(dev, cs, args, stream, peak, peak_kind, not args.no_cpu_baseline)
    dev.close()
    del cs
    base = None
    if not args.no_cpu_baseline:
        try:
            base = cpu_baseline(args.cpu_scale, name)
        except Exception as e:  # a missing toolchain must not hide the GPU number
            base = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": "failed: %s" % e}
    golden = m.pop("golden", None) or {"bit_exact": None}
    parity = {"full": "this workload's generator at 20 Mbp (tests/golden/full_s001.json) is bit-exact to the "
                      "reference's pipeline in the GPU tests; the full size has no reference run (hours on the host)",
              "pangenome": "this generator at 17 Mbp (tests/golden/pangenome_s002.json) is bit-exact in the GPU tests"}
    secondary = None
    if world == 1 and not args.no_secondary and name != "chromset":
        try:
            sm = measure(args, "chromset", 1.0, min(args.steps, 10), min(args.warmup, 3),
                         min(args.steps, args.e2e_steps), rank, world, local_rank, check=not args.no_check)
            sm.pop("dev").close()
            sm.pop("cs")
            sm.pop("autotune", None)
            secondary = {"workload": sm["config"]["workload"], "metric": METRIC, "unit": UNIT, **sm}
            if not args.no_cpu_baseline and not args.no_cpu_full_c2:
                # the reference's own pipeline on the same 2 x 100 Mbp input
                secondary["cpu_baseline"] = cpu_baseline(1.0, "chromset")
        except Exception as e:  # the secondary measurement must not hide the headline
            secondary = {"error": "%s: %s" % (type(e).__name__, e)}
        WL["name"] = name
    served = None
    if world == 1 and not args.no_serve:
        try:
            served = serve_compact(serve_measure(args))
        except Exception as e:  # the served measurement must not hide the plain number
            served = {"error": "%s: %s" % (type(e).__name__, e)}
    line = {
        "metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded generator, %s workload)" % name,
        "config": m["config"],
        "stage_ms": m["stage_ms"],
        "alloc_ms": m["alloc_ms"],
        "align_ms": m["align_ms"],
        "align_roofline": m["align_roofline"],
        "roofline": m["roofline"],
        "cpu_baseline": base,
        "e2e": m["e2e"],
        "gpu_launches": m["gpu_launches"],
        "clocks": m["clocks"],
        "bit_exact": golden.get("bit_exact"),
        "parity": golden if golden.get("bit_exact") is not None else parity.get(name, golden.get("reason")),
        "secondary": secondary,
        "gdb_ingest": ingest,
        "served_form": served,
        "autotune": m.get("autotune"),
    }
    emit(rank, line)


def run_serve(args) -> None:
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        line = serve_measure(args)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


def serve_measure(args) -> dict:
    """The served form beside the plain one on the same device and the same
    Poisson stream of query assemblies against one target: served = the
    target resident (ingested and indexed once), requests admitted as they
    arrive into `--serve-slots` concurrent slots; plain = each request alone,
    in arrival order, from the target's and the query's FASTA text (ingest,
    full index build, merge, alignment).  Latency = arrival to alignments on
    the host; throughput = GDB bases (target + query) of all requests / wall
    seconds from the first arrival to the last result.  Every served result
    is compared with the plain one (alignment records and trace bytes)."""
    from distributedpanga_b200 import build, pipeline, serve, synth
    build.build()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    sc = args.serve_scale
    contigs = synth.make_target(scale=sc)
    ttext = synth.fasta_bytes(contigs, "t")
    stream = synth.query_stream(contigs, args.serve_requests, args.serve_rate, int(1_000_000 * sc),
                                int(200_000_000 * sc), seed=31, median=2_000_000 * max(sc, 0.05))
    reqs = [serve.Request(k, synth.fasta_bytes(q, "q%d_" % k), arr, sum(len(c) for c in q))
            for k, (arr, q) in enumerate(stream)]
    t = time.monotonic()
    # one replica of the target per GPU; rank r serves the requests whose id
    # is congruent to r
    # with the record of its own Local_Alignment calls (the target's GDB
    # aligned once more, every call kept) for the requests' calls on target
    # contigs
    target = pipeline.Target(ttext, device=local_rank, reuse=True)
    target_s = time.monotonic() - t
    target_bases = target.bases
    big = max(reqs, key=lambda r: r.bases)
    # the device memory one request holds, measured on the largest one alone
    # (a context keeps its buffers): the served scheduler's charge per base
    import torch
    dp = pipeline.Device(local_rank)
    free0 = torch.cuda.mem_get_info(local_rank)[0]
    dp.gdb_ingest_fasta(ttext + big.text, tables=False)
    dp.index_build(want_entries=False)
    dp.merge(10)
    dp.align()
    held = free0 - torch.cuda.mem_get_info(local_rank)[0]
    dp.close()
    per_base = 1.1 * held / (target_bases + big.bases)
    srv = serve.Server(target, slots=args.serve_slots, bytes_per_base=per_base)
    dp = None

    def served(slot, r):
        # Server.execute with the host wall time of each call
        d, t0 = srv.devs[slot], time.monotonic()
        sizes = d.serve_load(target, r.text)
        t1 = time.monotonic()
        d.merge(srv.freq)
        t2 = time.monotonic()
        n = d.align()
        t3 = time.monotonic()
        al = d.alignments()
        t4 = time.monotonic()
        return {"nalign": n, "gdb_bases": int(sizes[5]), "query_bases": int(sizes[5]) - target.bases,
                "records": d.nrec, "alignments": al, "phases": [t1 - t0, t2 - t1, t3 - t2, t4 - t3],
                "reuse": d.reuse_stats()}

    def plain(slot, r):
        t0 = time.monotonic()
        dp.gdb_ingest_fasta(ttext + r.text, tables=False)
        dp.index_build(want_entries=False)
        t1 = time.monotonic()
        dp.merge(srv.freq)
        t2 = time.monotonic()
        n = dp.align()
        t3 = time.monotonic()
        al = dp.alignments()
        t4 = time.monotonic()
        return {"nalign": n, "gdb_bases": target_bases + r.bases, "query_bases": r.bases, "records": dp.nrec,
                "alignments": al, "phases": [t1 - t0, t2 - t1, t3 - t2, t4 - t3]}

    # The two forms one after the other, each holding the device alone (the
    # served form's slots and target are freed before the plain form runs).
    # Warm-up: the largest request on every slot (as many at once as the
    # memory budget admits), then on the plain context (kernels loaded, every
    # buffer at its largest size).
    srv.sched.run([serve.Request(k, big.text, 0.0, big.bases) for k in range(args.serve_slots)], served)
    clocks = ClockSampler(local_rank)
    clocks.start()
    res, summ = serve.serve_sharded(reqs, lambda mine: srv.sched.run(mine, served), rank, world)
    slots_admitted = max(1, max(len([q for q in res if q.admitted <= r.admitted < q.done]) for r in res)) if res else 0
    srv.close()
    target.close()
    dp = pipeline.Device(local_rank)
    plain(0, big)
    plain_sched = serve.Scheduler(1, 1 << 62, lambda r: 0)
    pres, psumm = serve.serve_sharded(reqs, lambda mine: plain_sched.run(mine, plain), rank, world)
    clk = clocks.stop()
    dp.close()
    if rank != 0:
        return None
    same = 0
    for a, b in zip(res, pres):
        if a.out["nalign"] == b.out["nalign"] and all(np.array_equal(x, y) for x, y in
                                                      zip(a.out["alignments"], b.out["alignments"])):
            same += 1
    line = {
        "metric": "served aligned Mbp/s (GDB bases of target + query per request / wall s) with p50/p99 request "
                  "latency, beside the plain form",
        "value": round(summ["gdb_mbp_per_s"], 2), "unit": "Mbp/s", "higher_is_better": True, "n_gpus": world,
        "scaling": "strong",
        "data": "synthetic (seeded)", "dtype": "u8",
        "config": {"workload": "serve: resident target of %d Mbp (chromset generator), %d Poisson requests at "
                               "%.1f/s, query sizes log-uniform %.1f-%.1f Mbp, divergence 0.5-5%%; k=40, FREQ=10"
                               % (round(target.bases / 1e6), len(reqs), args.serve_rate, 1 * sc, 200 * sc),
                   "slots": args.serve_slots, "max_requests_in_flight": slots_admitted,
                   "device_bytes_per_request_base": round(per_base / 1.1, 1),
                   "target_contigs": target.ncontig,
                   "parallelism": "replicas%d: one resident target per GPU, requests sharded by id" % world,
                   "target_build_s": round(target_s, 3)},
        "served": {k: round(v, 4) if isinstance(v, float) else v for k, v in summ.items()},
        "plain": {k: round(v, 4) if isinstance(v, float) else v for k, v in psumm.items()},
        "served_over_plain": round(summ["gdb_mbp_per_s"] / psumm["gdb_mbp_per_s"], 3),
        "bit_exact_requests": "%d/%d" % (same, len(reqs)),
        "call_record": {"requests_using_it": sum(1 for r in res if r.out["reuse"]["used"]),
                        "calls_from_record": sum(r.out["reuse"]["calls_from_record"] for r in res),
                        "calls": sum(r.out["reuse"]["calls"] for r in res),
                        "not_used": sorted({r.out["reuse"]["not_used"] for r in res if not r.out["reuse"]["used"]}),
                        "target_build_s": round(target_s, 3)},
        "requests": [{"rid": r.rid, "query_mbp": round(q.bases / 1e6, 3), "arrival_s": round(r.arrival, 3),
                      "served_latency_s": round(r.latency, 3), "plain_latency_s": round(p.latency, 3),
                      "alignments": r.out["nalign"], "calls_from_record": r.out["reuse"]["calls_from_record"],
                      "calls": r.out["reuse"]["calls"],
                      "served_phases_s": [round(x, 3) for x in r.out["phases"]],
                      "plain_phases_s": [round(x, 3) for x in p.out["phases"]]}
                     for r, p, q in zip(res, pres, reqs)],
        "phases": "load+index (served: query ingest + union with the resident index; plain: ingest of both texts + "
                  "index build), adaptamer merge, alignment (diagonal sorts included), alignments to the host; "
                  "host wall seconds, overlapping between served slots",
        "clocks": clk,
    }
    return line


def serve_compact(m: dict) -> dict:
    """The served measurement as one object of the main line."""
    keep = ("p50_latency_s", "p99_latency_s", "gdb_mbp_per_s", "query_mbp_per_s", "wall_s")
    return {"metric": "aligned Mbp/s (GDB bases of target + query per request / wall s), served vs plain form",
            "value": m["value"], "unit": "Mbp/s", "workload": m["config"]["workload"],
            "slots": m["config"]["slots"], "served": {k: m["served"][k] for k in keep},
            "plain": {k: m["plain"][k] for k in keep}, "served_over_plain": m["served_over_plain"],
            "bit_exact_requests": m["bit_exact_requests"], "call_record": m["call_record"], "clocks": m["clocks"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="full", choices=sorted(WORKLOADS),
                    help="full (2 x 1 Gbp, the default), chromset (2 x 100 Mbp) or pangenome (17 x 50 Mbp)")
    ap.add_argument("--scale", type=float, default=1.0, help="workload scale (1.0 = the workload's full size)")
    ap.add_argument("--ref-scale", type=float, default=None,
                    help="the reference arm's per-step sample of the generator (default %s)" % REF_SCALE)
    ap.add_argument("--cpu-scale", type=float, default=None,
                    help="the cpu_baseline sample of the generator (default %s)" % CPU_SCALE)
    ap.add_argument("--no-cpu-full-c2", action="store_true",
                    help="skip timing the reference on the whole 2 x 100 Mbp workload (the secondary's cpu_baseline; "
                         "about 1.5 min plus GIXmake)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--entries", action="store_true",
                    help="also write the reference-format k-mer table entries in every step (N x E bytes of HBM)")
    ap.add_argument("--e2e-steps", type=int, default=3, help="end-to-end steps (after one warm-up), at most --steps")
    ap.add_argument("--no-check", action="store_true", help="skip the comparison with the reference's digests")
    ap.add_argument("--no-secondary", action="store_true", help="skip the 2 x 100 Mbp secondary measurement")
    ap.add_argument("--no-ingest", action="store_true", help="skip the FASTA ingest measurement")
    ap.add_argument("--digit-bits", type=int, default=0,
                    help="with --profile-stage index: the index sort's first digit width (0 automatic, 18..22)")
    ap.add_argument("--align-build", type=int, default=0,
                    help="with --profile-stage align: the alignment kernel's build (0 automatic, 2 to 5)")
    ap.add_argument("--profile-stage", choices=["index", "ingest", "serve", "align", "diag"], default=None,
                    help="run only this stage (warmup + steps calls) and print its device times; for profiling")
    ap.add_argument("--serve", action="store_true",
                    help="measure the served form (resident target, concurrent requests) beside the plain one")
    ap.add_argument("--serve-scale", type=float, default=1.0,
                    help="served workload scale: target 1 Gbp x S, queries 1-200 Mbp x S (default 1.0)")
    ap.add_argument("--serve-requests", type=int, default=12)
    ap.add_argument("--serve-rate", type=float, default=2.0, help="request arrivals per second (Poisson)")
    ap.add_argument("--serve-slots", type=int, default=3)
    ap.add_argument("--autotune", action="store_true",
                    help="time the digit width, aligner build and band-range size on the workload first "
                         "(untimed) and run with the fastest")
    ap.add_argument("--no-serve", action="store_true",
                    help="leave the served-form measurement out of the main line")
    args = ap.parse_args()
    if args.serve:
        run_serve(args)
        return
    WL["name"] = args.workload
    if args.ref_scale is None:
        args.ref_scale = REF_SCALE[args.workload]
    if args.cpu_scale is None:
        args.cpu_scale = CPU_SCALE[args.workload]
    if args.profile_stage:
        run_profile_stage(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
