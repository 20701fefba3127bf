"""BASELINE config 5 at full size: 1024 templates over three series lengths
(2^20, 3*2^20, 2^22 in ratio 4:2:1) in one captured graph, thresholds at 5 and 7
sigma-equivalent.  Every template's candidates against the CPU oracle pipeline
(run in parallel host processes) and the toplist of each series against the
oracle's toplist."""
import multiprocessing as mp
import os

import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import shard, synth

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
THRESH_RTOL = 1e-5
_W = {}


def _init(series):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "boinc-einstein-bpr4-v3d_b200")]
    from oracle import oracle as O
    _W["O"], _W["series"] = O, series


def _oracle_candidates(args):
    s, pbytes = args
    O = _W["O"]
    p = O.Params.from_buffer_copy(pbytes)
    return O.pipeline(_W["series"][s], p)["candidates"]


def _same(got, ref, p):
    kg = {(int(b), int(l)): float(v) for b, l, v in zip(got["bin"], got["level"], got["power"])}
    kr = {(int(b), int(l)): float(v) for b, l, v in zip(ref["bin"], ref["level"], ref["power"])}
    for k in set(kg) | set(kr):
        thr = float(p.threshold[k[1]])
        if k in kg and k in kr:
            assert abs(kg[k] - kr[k]) <= 2e-4 * (1 + abs(kr[k])), k
        else:
            v = kg.get(k, kr.get(k))
            assert abs(v - thr) <= THRESH_RTOL * thr, (k, v, thr)


def test_uneven_bank_config5(oracle):
    wl = synth.config5(1024)
    ctx = mp.get_context("spawn")
    with ctx.Pool(max(2, min(32, os.cpu_count() or 2)), initializer=_init, initargs=(wl.series,)) as pool:
        ref = pool.map(_oracle_candidates, [(int(s), bytes(p)) for s, p in zip(wl.series_of, wl.templates)],
                       chunksize=4)
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    for s, x in enumerate(wl.series):
        bank.set_series(s, x)
    got, counts, status = bank.run(wl.templates, wl.series_of)
    assert not status.any()
    assert sum(len(c) for c in got) > 100
    for g, r, p in zip(got, ref, wl.templates):
        _same(g, r, p)
    for s in range(len(wl.series)):
        idx = [t for t in range(len(wl.templates)) if wl.series_of[t] == s]
        temps = [wl.templates[t] for t in idx]
        orbs = [wl.orbits[t] for t in idx]
        top = shard.fold_toplist(B.Toplist(), temps, orbs, [got[t] for t in idx]).final()
        rtop = shard.fold_toplist(oracle.Toplist(), temps, orbs, [ref[t] for t in idx]).final()
        assert len(top) == len(rtop)
        for a, b in zip(top, rtop):
            assert (a["bin"], a["harmonics"], a["period"], a["tau"], a["psi"]) == \
                   (b["bin"], b["harmonics"], b["period"], b["tau"], b["psi"])
    bank.close()
