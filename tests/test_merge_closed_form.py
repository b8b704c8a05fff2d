"""The closed form the GPU merge kernel uses, checked on the CPU against the
oracle's restatement of the reference's sequential walk
(src/fastga_pipeline.c:245-412).

Closed form, per table entry i with lcp[] the LCP-to-predecessor sequence:
plen = max(lcp[i], lcp[i+1]); the run is the maximal [s, t) around i with
lcp[r] >= plen for s < r < t; i emits a seed to every other member iff
t - s < FREQ (and plen >= 12)."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_case
from helpers import canonical_rows


def closed_form_merge(srt, posb, ctgb, freq):
    lcp = srt[:, 0].astype(np.int64)
    n = len(lcp)
    pay = srt[:, 12:]
    sbit = 0x80
    out_n, out_c = [], []
    for i in range(n):
        plen = max(lcp[i], lcp[i + 1] if i + 1 < n else 0)
        if plen < 12:
            continue
        s = i
        while s > 0 and lcp[s] >= plen:
            s -= 1
        t = i + 1
        while t < n and lcp[t] >= plen:
            t += 1
        if t - s >= freq:
            continue
        a = pay[i].copy()
        isign = a[-1] & sbit
        a[-1] &= 0x7F
        for j in range(s, t):
            if j == i:
                continue
            row = np.concatenate([[plen], a, pay[j]]).astype(np.uint8)
            (out_n if (pay[j][-1] & sbit) == isign else out_c).append(row)
    sb = 1 + 2 * (posb + ctgb)
    mk = lambda L: np.array(L, dtype=np.uint8).reshape(-1, sb)
    return mk(out_n), mk(out_c)


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_closed_form_equals_sequential_walk(oracle, case):
    cs, dig = load_case(case)
    posb, ctgb = dig["posb"], dig["ctgb"]
    srt = oracle.sort_records(oracle.extract(cs, posb, ctgb))
    ent, cum, _ = oracle.build_adapter(srt, posb, ctgb)
    ns, css, _, _ = oracle.merge(ent, cum, posb, ctgb, 10, cs.ncontig)
    cn, cc = closed_form_merge(srt, posb, ctgb, 10)
    # same entry order on both sides, so the streams are equal, not just the multisets
    assert np.array_equal(cn, ns)
    assert np.array_equal(cc, css)
