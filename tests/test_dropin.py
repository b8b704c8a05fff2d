"""The reference's own driver, unchanged (src/pga-mpi-merge.c), linked with
the B200 drop-in stages (distributedpanga_b200/dropin/pga_dropin.c over
libpga_b200.so) in place of src/extract.c, src/sort.c, src/kmer_adapter.c and
src/fastga_pipeline.c (oracle/Makefile `dropin`).  Run on a golden case's
GDB, its .1aln must be the stock build's record stream, and its own stage
log must report the stock build's record and seed counts."""
import gzip
import os
import re
import tempfile

import pytest

from conftest import GOLDEN, ROOT, load_case

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "oracle", "_ref", "pga-mpi-merge-b200")


@pytest.mark.parametrize("case", ["small_s002", "edge_mix", "many_contigs", "chromset_s0005", "small_full"])
def test_reference_driver_on_b200_stages(case):
    import subprocess
    from distributedpanga_b200 import synth
    from oracle import binding as B
    if not (os.path.exists(DRIVER) and B.ref_available()):
        pytest.skip("oracle/_ref not built (make -C oracle ref dropin)")
    cs, dig = load_case(case)
    contigs = [cs.contig(i) for i in range(cs.ncontig)]
    with tempfile.TemporaryDirectory() as tmp:
        fa = os.path.join(tmp, "g.fa")
        stem = os.path.join(tmp, "g")
        synth.write_fasta(fa, contigs)
        B.ref_make_gdb(fa, stem)
        out = B.ref_run(stem, tmp, threads=1, driver="pga-mpi-merge-b200")
        log = open(out["log"]).read()
        aln = subprocess.run([os.path.join(B.REF_DIR, "alndump"), out["aln"]], check=True, capture_output=True,
                             text=True).stdout
    o1 = dict(re.findall(r"(\w+)=([0-9.]+)", log.split("[o1-0]")[1].split("\n")[0]))
    pr = dict(re.findall(r"(\w+)=([0-9.]+)", log.split("[pr1]")[1].split("\n")[0]))
    assert int(o1["records"]) == dig["index"]["count"]
    assert int(o1["slice_records"]) == dig["index"]["count"]
    assert int(pr["seeds_n"]) == dig["seeds"]["n_count"] and int(pr["seeds_c"]) == dig["seeds"]["c_count"]
    mine = [" ".join(x.split()) for x in aln.split("\n") if x.strip() and not x.startswith("#")]
    ref = [" ".join(x.split()) for x in gzip.open(os.path.join(GOLDEN, case + ".aln.txt.gz"), "rt").read().split("\n")
           if x.strip()]
    assert len(mine) == dig["aln"]["count"]
    assert mine == ref
