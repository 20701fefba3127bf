"""Device toplist pre-filter of the bank (brp_cuda_bank_set_toplist_filter):
the kept candidates of every template are a subset of its full list, and
folding them into the toplist (src/workload.cpp:126-159) in bank order gives
byte-identical final rows to folding every candidate -- on one series with
far more than 100 distinct bins per level, and per series on a bank of three
lengths.  Turning the filter off again returns every candidate."""
import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import synth

pytestmark = pytest.mark.gpu
CAP = 8192


def run(bank, wl):
    flat, offs, counts, status = bank.run_flat(B.Bank.params_array(wl.templates), wl.series_of)
    assert not status.any()
    return [flat[offs[t]:offs[t + 1]].copy() for t in range(len(wl.templates))]


def finals(wl, lists):
    out = {}
    for s in range(len(wl.series)):
        idx = [t for t in range(len(wl.templates)) if wl.series_of[t] == s]
        top = B.Toplist().fold([wl.templates[t] for t in idx], [wl.orbits[t] for t in idx], [lists[t] for t in idx])
        out[s] = top.final()
    return out


def keys(c):
    return set(zip(c["bin"].tolist(), c["level"].tolist(), c["power"].view(np.uint32).tolist()))


@pytest.mark.parametrize("name,lengths,counts,pulsars", [
    ("one-series", [1 << 20], [96], [3]),
    ("three-lengths", [1 << 18, 3 << 17, 1 << 19], [40, 24, 16], [2, 1, 2]),
])
def test_filter_keeps_the_final_toplist(name, lengths, counts, pulsars):
    # thresholds at 4 sigma: noise candidates in every template, hundreds to
    # thousands of distinct bins per level across the bank
    wl = synth.bank_workload(name, lengths, counts, pulsars, seed=41, sigmas=(4.0,))
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), CAP)
    for s, x in enumerate(wl.series):
        bank.set_series(s, x)
    full = run(bank, wl)
    bank.set_toplist_filter(100)
    kept = run(bank, wl)
    kept2 = run(bank, wl)  # graph replay with the filter state of the previous run cleared
    bank.set_toplist_filter(0)
    again = run(bank, wl)
    bank.close()
    n_full = sum(len(c) for c in full)
    n_kept = sum(len(c) for c in kept)
    for f, k, k2, a in zip(full, kept, kept2, again):
        assert keys(k) <= keys(f)
        assert np.array_equal(k, k2)
        assert np.array_equal(a, f)
        assert np.array_equal(k, np.sort(k, order=["level", "bin"]))
    fa, fk = finals(wl, full), finals(wl, kept)
    for s in fa:
        assert fa[s].tobytes() == fk[s].tobytes()
        assert len(fa[s]) > 0
    print("%s: %d of %d candidates kept" % (name, n_kept, n_full))
    assert n_kept < n_full // 2
