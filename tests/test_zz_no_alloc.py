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


def test_noalloc_matches_allocating_entry_point(dev, oracle):
    import torch
    from distributedpanga_b200 import pipeline
    L = pipeline.load_library()
    f = L.pga_reimport_sort_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int, C.c_void_p,
                  C.c_void_p, C.c_void_p]
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
    from distributedpanga_b200 import pipeline
    L = pipeline.load_library()
    f = L.pga_reimport_sort_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int, C.c_void_p,
                  C.c_void_p, C.c_void_p]
    sb = 1 + 2 * (3 + 1)
    n = (1 << 18) + 1
    s_dev = torch.zeros(n * sb, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    off = torch.zeros(8, dtype=torch.int64, device="cuda")
    rc = f(s_dev.data_ptr(), n * sb, 3, 1, 0, 4, 1000, 3, out.data_ptr(), off.data_ptr(), None)
    assert rc == 4  # PGA_ERR_LIMIT, before any GPU work
