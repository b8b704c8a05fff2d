"""The autotuner's selection logic on the host, with a fake device whose
calls advance a fake clock by a cost that depends on the knob settings."""
from __future__ import annotations

import pytest

from distributedpanga_b200 import autotune


class FakeDev:
    def __init__(self, index_cost, align_cost):
        self.t = 0.0
        self.bits = self.build = self.ranges = 0
        self.long = autotune.LONG_WAVES_DEFAULT
        self.index_cost, self.align_cost = index_cost, align_cost
        self.calls = []

    def clock(self):
        return self.t

    def set_digit_bits(self, b):
        self.bits = b

    def set_build(self, b):
        self.build = b

    def set_ranges(self, r):
        self.ranges = r

    def set_long_waves(self, w):
        self.long = w

    def index_build(self, want_entries=True):
        self.t += self.index_cost(self.bits)
        self.calls.append(("index", self.bits))
        return 100

    def merge(self, freq):
        return 300_000_000, 100_000_000

    def align(self):
        self.t += self.align_cost(self.build, self.ranges) - (0.05 if self.long == 10000 else 0.0)
        self.calls.append(("align", self.build, self.ranges))
        return 5


def test_picks_fastest_and_restores_defaults():
    d = FakeDev(lambda b: abs(b - 20) + 1.0, lambda b, r: (1.0 if b == 3 else 2.0) + (0.5 if r == -1 else 0.1 * (r > 2000)))
    t = autotune.Tuner(d, repeats=3, clock=d.clock)
    cfg = t.tune()
    assert cfg["digit_bits"] == 20
    assert cfg["align_build"] == 3
    # never-split costs 0.5, sizes above 2000 seeds 0.1: the automatic size
    # (844 here) ties with its half and comes first
    assert cfg["range_seeds"] == autotune.auto_range_seeds(400_000_000) == 844
    assert cfg["long_waves"] == 10000
    assert (d.bits, d.build, d.ranges, d.long) == (0, 0, 0, autotune.LONG_WAVES_DEFAULT)  # defaults again
    assert sum(1 for c in d.calls if c[0] == "index") == 3 * len(autotune.DIGIT_BITS) + 1
    assert set(t.times["digit_bits"]) == set(autotune.DIGIT_BITS)


def test_choose_uses_median():
    assert autotune.choose({"a": [1.0, 9.0, 9.0], "b": [5.0, 5.0, 5.0], "c": [0.1, 6.0, 6.0]}) == "b"
    assert autotune.choose({"x": [2.0], "y": [2.0]}) == "x"


def test_range_candidates():
    assert autotune.auto_range_seeds(10) == 256
    s = 160 * autotune.AUTO_WARPS * 1000
    assert autotune.range_candidates(s) == (-1, 1000, 500, 2000)
    assert autotune.range_candidates(10) == (-1, 256, 512)


def test_apply_and_cache(tmp_path):
    d = FakeDev(lambda b: 1.0, lambda b, r: 1.0)
    autotune.apply(d, {"digit_bits": 19, "align_build": 2, "range_seeds": -1, "long_waves": 0})
    assert (d.bits, d.build, d.ranges, d.long) == (19, 2, -1, 0)
    autotune.apply(d, {})
    assert (d.bits, d.build, d.ranges, d.long) == (0, 0, 0, autotune.LONG_WAVES_DEFAULT)
    p = str(tmp_path / "tune.json")
    c = autotune.TuneCache(p)
    sig = autotune.signature(200_123_456, 300, 1_234_567_890)
    assert sig == "b20e7-c30e1-s12e8"
    assert c.get(sig) is None
    c.put(sig, {"digit_bits": 18})
    assert autotune.TuneCache(p).get(sig) == {"digit_bits": 18}
    assert autotune.signature(42, 7, 0) == "b42-c7-s0"


@pytest.mark.gpu
def test_tuned_configuration_keeps_reference_alignments(dev):
    """Tuning on a golden case (every candidate runs) and running with the
    chosen configuration gives the reference's alignments."""
    import gzip
    import os
    from conftest import GOLDEN, load_case
    from distributedpanga_b200.pipeline import alignment_lines
    cs, dig = load_case("chromset_s0005")
    dev.gdb_load(cs)
    tu = autotune.Tuner(dev, repeats=1, freq=dig["freq_cutoff"])
    cfg = tu.tune()
    assert cfg["digit_bits"] in autotune.DIGIT_BITS and cfg["align_build"] in autotune.ALIGN_BUILDS
    try:
        autotune.apply(dev, cfg)
        dev.index_build(want_entries=False)
        dev.merge(dig["freq_cutoff"])
        dev.align()
        got = [" ".join(l.split()) for l in alignment_lines(*dev.alignments()) if l.strip()]
    finally:
        autotune.apply(dev, {})
    ref = [" ".join(l.split()) for l in gzip.open(os.path.join(GOLDEN, "chromset_s0005.aln.txt.gz"), "rt")
           .read().split("\n") if l.strip()]
    assert got == ref
