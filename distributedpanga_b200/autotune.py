"""Autotuner for the alignment path's launch parameters.

Four knobs change how the device does the work but never what it computes
(each is covered by a parity test that runs the path at several settings):

* ``digit_bits`` -- width of the index sort's first-level digit
  (``pga_index_set_digit_bits``, 18..22).  Wider digits mean more, smaller
  shared-memory sorts and more scatter fronts;
* ``align_build`` -- which build of the alignment kernel runs
  (``pga_align_set_build``: 2 CTAs per SM at 255 registers, 3 at 168, 4 at
  128 or 5 at 96);
* ``range_seeds`` -- how large pairs are cut into band ranges that different
  warps align (``pga_align_set_ranges``: -1 never, or a size in seeds; the
  automatic size is max(256, seeds / (160 x 2960 warps)));
* ``long_waves`` -- after how many wave steps a Local_Alignment call keeps
  its SM to itself (``pga_align_set_long_waves``; 0 never, -1 automatic).

``Tuner.tune`` times every candidate on the GDB loaded in a context (the
workload itself, or a sample of it): the index knob with the index build
alone, the alignment knobs with the alignment (diagonal sorts included)
after one adaptamer merge, the long-call threshold last, with the chosen
build and range size set.  Each candidate runs ``repeats`` times and the
one with the lowest median wins.  ``TuneCache`` keeps the choices in a JSON
file keyed by the workload's signature (bases, contigs, seeds, each to two
significant digits) so that a recurring workload is tuned once.
"""
from __future__ import annotations

import json
import math
import os
import statistics
import time

DIGIT_BITS = (18, 19, 20, 21, 22)
ALIGN_BUILDS = (2, 3, 4, 5)
LONG_WAVES = (0, 10000, 20000, 40000)
LONG_WAVES_DEFAULT = -1        # automatic: 20000 for the two-CTA build, off for the three-CTA one
AUTO_WARPS = 148 * 20          # the alignment launch's task warps (pga_align's work spaces)


def auto_range_seeds(all_seeds: int) -> int:
    return max(256, all_seeds // (160 * AUTO_WARPS))


def range_candidates(all_seeds: int) -> tuple:
    """-1 (never split), the automatic size, half and twice it."""
    a = auto_range_seeds(all_seeds)
    return tuple(dict.fromkeys((-1, a, max(256, a // 2), 2 * a)))


def choose(times: dict):
    """The key whose list of durations has the lowest median (ties: the first)."""
    best, bt = None, math.inf
    for k, v in times.items():
        m = statistics.median(v)
        if m < bt:
            best, bt = k, m
    return best


def signature(bases: int, contigs: int, seeds: int) -> str:
    def two(x):
        x = int(x)
        if x < 100:
            return str(x)
        e = int(math.floor(math.log10(x))) - 1
        return "%de%d" % (round(x / 10 ** e), e)
    return "b%s-c%s-s%s" % (two(bases), two(contigs), two(seeds))


class Tuner:
    """Times the knobs on `dev` (a pipeline.Device with a GDB loaded)."""

    def __init__(self, dev, repeats: int = 3, freq: int = 10, clock=time.perf_counter):
        self.dev = dev
        self.repeats = repeats
        self.freq = freq
        self.clock = clock
        self.times = {}

    def _time(self, fn) -> list:
        out = []
        for _ in range(self.repeats):
            t = self.clock()
            fn()
            out.append(self.clock() - t)
        return out

    def tune_index(self, candidates=DIGIT_BITS) -> int:
        d = self.dev
        times = {}
        try:
            for b in candidates:
                d.set_digit_bits(b)
                times[b] = self._time(lambda: d.index_build(want_entries=False))
        finally:
            d.set_digit_bits(0)
        self.times["digit_bits"] = times
        return choose(times)

    def tune_align(self, builds=ALIGN_BUILDS, ranges=None) -> tuple:
        d = self.dev
        d.index_build(want_entries=False)
        ns, cs = d.merge(self.freq)
        if ranges is None:
            ranges = range_candidates(ns + cs)
        times = {}
        try:
            for b in builds:
                d.set_build(b)
                for r in ranges:
                    d.set_ranges(r)
                    times[(b, r)] = self._time(d.align)
        finally:
            d.set_build(0)
            d.set_ranges(0)
        self.times["align"] = {"%d/%d" % k: v for k, v in times.items()}
        self.seeds = ns + cs
        return choose(times)

    def tune_long(self, build: int, rs: int, candidates=LONG_WAVES) -> int:
        d = self.dev
        times = {}
        try:
            d.set_build(build)
            d.set_ranges(rs)
            for w in candidates:
                d.set_long_waves(w)
                times[w] = self._time(d.align)
        finally:
            d.set_build(0)
            d.set_ranges(0)
            d.set_long_waves(LONG_WAVES_DEFAULT)
        self.times["long_waves"] = times
        return choose(times)

    def tune(self) -> dict:
        bits = self.tune_index()
        build, rs = self.tune_align()
        lw = self.tune_long(build, rs)
        return {"digit_bits": bits, "align_build": build, "range_seeds": rs, "long_waves": lw}


def apply(dev, cfg: dict) -> None:
    """Sets a tuned configuration on a context (keys missing: automatic)."""
    dev.set_digit_bits(int(cfg.get("digit_bits", 0)))
    dev.set_build(int(cfg.get("align_build", 0)))
    dev.set_ranges(int(cfg.get("range_seeds", 0)))
    dev.set_long_waves(int(cfg.get("long_waves", LONG_WAVES_DEFAULT)))


class TuneCache:
    """Tuned configurations on disk, by workload signature."""

    def __init__(self, path: str):
        self.path = path
        self.data = {}
        if os.path.exists(path):
            with open(path) as f:
                self.data = json.load(f)

    def get(self, sig: str):
        return self.data.get(sig)

    def put(self, sig: str, cfg: dict) -> None:
        self.data[sig] = cfg
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)
