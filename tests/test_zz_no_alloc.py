"""The diagonal sort entry point that allocates no device memory.

It exists for callers that may not call cudaMalloc themselves -- a program
that lives inside another framework's device memory pool, such as PyTorch's
caching allocator or a serving runtime's arena, and owns only the buffers
that pool gives it.  Here torch plays that framework: it owns the seed,
output and panel buffers, and the library's fixed scratch array does the
rest.  The result must equal the allocating entry point's (pga_reimport_sort)
byte for byte, on two calls in a row (the scratch keeps the previous call's
contents between them).

This file is collected last so that a run stopping at the first failure has
run every other test before it."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_case

pytestmark = pytest.mark.gpu


def _seeds(oracle, case):
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    srt = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    ent, cum, _ = oracle.build_adapter(srt, posb, ctgb)
    ns, css, _, _ = oracle.merge(ent, cum, posb, ctgb, 10, cs.ncontig)
    return cs, dig, ns, css


def _entry():
    from distributedpanga_b200 import pipeline
    L = pipeline.load_library()
    f = L.pga_reimport_sort_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int, C.c_void_p,
                  C.c_void_p, C.c_void_p]
    return f


def _call(f, seeds, posb, ctgb, comp, ncontig, amxpos, dbyte, off_fill=0):
    """One call on torch-owned device buffers; returns (rc, records, panel offsets)."""
    import torch
    swide = 2 * dbyte + ctgb + 2
    flat = np.ascontiguousarray(seeds).reshape(-1)
    s_dev = torch.from_numpy(flat).to("cuda") if flat.size else torch.zeros(1, dtype=torch.uint8, device="cuda")
    n = seeds.shape[0]
    out = torch.zeros(max(1, n * swide), dtype=torch.uint8, device="cuda")
    off = torch.full((ncontig + 1,), off_fill, dtype=torch.int64, device="cuda")
    rc = f(s_dev.data_ptr(), flat.size, posb, ctgb, comp, ncontig, amxpos, dbyte, out.data_ptr(), off.data_ptr(),
           torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()[: n * swide].reshape(n, swide), off.cpu().numpy()


def test_noalloc_matches_golden_panels(dev, oracle):
    """The reference's own sorted diagonal panels (golden digests), N then C."""
    from helpers import check_diag
    f = _entry()
    cs, dig, ns, css = _seeds(oracle, "small_s002")
    for comp, u, seeds in ((0, "N", ns), (1, "C", css)):
        rc, got, off = _call(f, seeds, dig["posb"], dig["ctgb"], comp, cs.ncontig, cs.maxctg, dig["dbyte"])
        assert rc == 0
        check_diag(got, off, u, dig)


def _random_seeds(rng, n, ncontig, clen, posb, ctgb, comp):
    """n seeds of the reference layout [plen][A pos][A contig][B pos][B contig|strand]
    with positions inside random contigs: A forward, B's strand bit = comp."""
    sb = 1 + 2 * (posb + ctgb)
    a = rng.integers(0, ncontig, n)
    b = rng.integers(0, ncontig, n)
    ap = (rng.random(n) * clen[a]).astype(np.int64)
    bp = (rng.random(n) * clen[b]).astype(np.int64)
    s = np.zeros((n, sb), np.uint8)
    s[:, 0] = rng.integers(12, 41, n)
    for k in range(posb):
        s[:, 1 + k] = (ap >> (8 * k)) & 0xff
        s[:, 1 + posb + ctgb + k] = (bp >> (8 * k)) & 0xff
    bc = b | (comp << (8 * ctgb - 1))
    for k in range(ctgb):
        s[:, 1 + posb + k] = (a >> (8 * k)) & 0xff
        s[:, 1 + 2 * posb + ctgb + k] = (bc >> (8 * k)) & 0xff
    return s


def test_noalloc_at_the_seed_limit(dev, oracle):
    """Exactly 262,144 seeds (the fixed scratch's limit: every offset of the
    array in use) over 300 contigs of up to 4 Mbp, so that nearly every key
    byte differs and every radix pass runs; twice in a row, N then C, each
    against the allocating entry point and the oracle."""
    f = _entry()
    rng = np.random.default_rng(8)
    ncontig, posb, ctgb = 300, 3, 2
    clen = rng.integers(1000, 4_000_000, ncontig)
    amxpos = int(clen.max())
    dbyte = 1
    while (1 << (8 * dbyte)) < 2 * amxpos:
        dbyte += 1
    for comp in (0, 1):
        seeds = _random_seeds(rng, 1 << 18, ncontig, clen, posb, ctgb, comp)
        rc, got, off = _call(f, seeds, posb, ctgb, comp, ncontig, amxpos, dbyte)
        assert rc == 0
        want, want_off = dev.reimport_sort(seeds, posb, ctgb, comp, ncontig, amxpos, dbyte)
        assert np.array_equal(got, want) and np.array_equal(off, want_off)
        owant, owant_off = oracle.reimport_sort(seeds, posb, ctgb, comp, ncontig, amxpos, dbyte)
        assert np.array_equal(got, owant) and np.array_equal(off, owant_off)


def test_noalloc_no_seeds(dev, oracle):
    """len = 0 after a call that left the scratch full: every panel offset 0."""
    f = _entry()
    cs, dig, ns, _ = _seeds(oracle, "small_s002")
    rc, _, _ = _call(f, ns, dig["posb"], dig["ctgb"], 0, cs.ncontig, cs.maxctg, dig["dbyte"])
    assert rc == 0
    rc, got, off = _call(f, ns[:0], dig["posb"], dig["ctgb"], 0, cs.ncontig, cs.maxctg, dig["dbyte"], off_fill=7)
    assert rc == 0 and got.shape[0] == 0
    assert np.array_equal(off, np.zeros(cs.ncontig + 1, np.int64))


def test_noalloc_rejects_partial_seed(dev):
    """A length that is not a whole number of seeds is an argument error, in
    this entry point and in the allocating one."""
    from distributedpanga_b200 import pipeline
    f = _entry()
    posb, ctgb = 3, 1
    sb = 1 + 2 * (posb + ctgb)
    seeds = np.zeros((10, sb), np.uint8)
    import torch
    s_dev = torch.zeros(10 * sb, dtype=torch.uint8, device="cuda")
    out = torch.zeros(10 * 8, dtype=torch.uint8, device="cuda")
    off = torch.zeros(5, dtype=torch.int64, device="cuda")
    assert f(s_dev.data_ptr(), 10 * sb - 1, posb, ctgb, 0, 4, 1000, 2, out.data_ptr(), off.data_ptr(), None) == 2
    with pytest.raises(pipeline.PgaError):
        rc = dev.L.pga_reimport_sort(dev.h, seeds.ctypes.data_as(C.c_void_p), seeds.size - 1, posb, ctgb, 0, 4,
                                     1000, 2, np.zeros(80, np.uint8).ctypes.data_as(C.c_void_p),
                                     np.zeros(5, np.int64))
        dev._ck(rc, "reimport_sort")


def test_noalloc_matches_allocating_entry_point(dev, oracle):
    import torch
    f = _entry()
    cs, dig, ns, css = _seeds(oracle, "small_s002")
    posb, ctgb, dbyte, swide = dig["posb"], dig["ctgb"], dig["dbyte"], dig["swide"]
    stream = torch.cuda.current_stream()
    # two calls in a row: N seeds then C seeds (each then checked against the allocating path)
    for comp, seeds in ((0, ns), (1, css), (0, ns)):
        want, want_off = dev.reimport_sort(seeds, posb, ctgb, comp, cs.ncontig, cs.maxctg, dbyte)
        s_dev = torch.from_numpy(np.ascontiguousarray(seeds).reshape(-1)).to("cuda")
        out = torch.zeros(seeds.shape[0] * swide, dtype=torch.uint8, device="cuda")
        off = torch.zeros(cs.ncontig + 1, dtype=torch.int64, device="cuda")
        rc = f(s_dev.data_ptr(), seeds.size, posb, ctgb, comp, cs.ncontig, cs.maxctg, dbyte, out.data_ptr(),
               off.data_ptr(), stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(-1, swide)
        assert np.array_equal(got, want)
        assert np.array_equal(off.cpu().numpy(), want_off)


def test_noalloc_rejects_too_many_seeds(dev):
    import torch
    f = _entry()
    sb = 1 + 2 * (3 + 1)
    n = (1 << 18) + 1
    s_dev = torch.zeros(n * sb, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    off = torch.zeros(8, dtype=torch.int64, device="cuda")
    rc = f(s_dev.data_ptr(), n * sb, 3, 1, 0, 4, 1000, 3, out.data_ptr(), off.data_ptr(), None)
    assert rc == 4  # PGA_ERR_LIMIT, before any GPU work
