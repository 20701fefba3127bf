"""Host-side logic of the product (template constants, search parameters,
toplist) against the CPU oracle and, where built, the reference's own
compiled code.  No GPU needed: these are host functions of libbrp_cuda.so."""
import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import synth

CASES = [
    (65536, 65536 - 17, 0.002, 120.0, 0.3, 256e-6),
    (65536, 65536 - 17, 0.3, 3600.0, 1.1, 128e-6),
    (1 << 22, (1 << 22) - 17, 1.7, 11 * 3600.0, 0.4, 128e-6),
    (3 << 21, 3 << 21, 3.0, 3600.0, -5.0, 128e-6),
    (64, 47, 0.0, 10.0, 0.0, 1e-3),
    (96, 64, 1e-3, 1.0, 6.2, 1e-3),
]


@pytest.mark.parametrize("case", CASES)
def test_parameters_match_oracle(oracle, case):
    p = B.parameters(*case)
    q = oracle.parameters(*case)
    assert bytes(p) == bytes(q)
    assert bytes(B.production(p)) == bytes(oracle.production(q))


@pytest.mark.parametrize("bad", [(63, 60, 0.1, 1.0, 0.0, 1e-3), (100, 90, 0.1, 1.0, 0.0, 1e-3),
                                 (64, 65, 0.1, 1.0, 0.0, 1e-3), (64, 60, -1.0, 1.0, 0.0, 1e-3),
                                 (64, 60, 0.1, 0.0, 0.0, 1e-3), (64, 60, 0.1, 1.0, float("nan"), 1e-3)])
def test_parameters_reject_like_reference(oracle, bad):
    with pytest.raises(B.BrpError):
        B.parameters(*bad)
    with pytest.raises(oracle.OracleError):
        oracle.parameters(*bad)


@pytest.mark.parametrize("orbit", [(3600.0, 0.3, 1.1), (86000.0, 2.9, 4.0), (20000.0, 0.0, 0.0)])
@pytest.mark.parametrize("obs", [(1 << 22, 1 << 22), (3 << 20, 3 << 20), (1 << 20, 900000)])
def test_search_parameters_match_oracle(oracle, orbit, obs):
    n, samples = obs
    for f0, fa, w in [(400.0, 0.08, 1000), (800.0, 0.01, 500), (50.0, 1e-6, 7)]:
        p = B.search_parameters(n, samples, 128.0, *orbit, f0, fa, w)
        q = oracle.search_parameters(n, samples, 128.0, *orbit, f0, fa, w)
        assert bytes(p) == bytes(q)


def test_search_parameters_match_reference(oracle):
    if not oracle.ref_available():
        pytest.skip("reference build absent (oracle/_ref)")
    rng = np.random.default_rng(5)
    for _ in range(20):
        P, tau, psi = synth.random_orbits(rng, 1)[0]
        p = B.search_parameters(1 << 22, 1 << 22, 128.0, P, tau, psi, 400.0, 0.08, 1000)
        r = oracle.ref_search_parameters(1 << 22, 1 << 22, 128.0, P, tau, psi, 400.0, 0.08, 1000)
        assert bytes(p) == bytes(r)


def test_sigma_false_alarm_thresholds():
    n = 1 << 20
    p5 = B.search_parameters(n, n, 128.0, 3600.0, 0.5, 0.1, 400.0, synth.sigma_false_alarm(n, 5.0), 1000)
    p7 = B.search_parameters(n, n, 128.0, 3600.0, 0.5, 0.1, 400.0, synth.sigma_false_alarm(n, 7.0), 1000)
    # level 0 threshold = -ln(p): 5 sigma tail 2.87e-7 -> 15.06, 7 sigma 1.28e-12 -> 27.4
    assert abs(p5.threshold[0] - 15.06) < 0.05
    assert abs(p7.threshold[0] - 27.38) < 0.05
    assert all(a < b for a, b in zip(p5.threshold, p7.threshold))


def _random_candidates(rng, p, count):
    bins = rng.integers(p.window, p.fundamental, count)
    levels = rng.integers(0, 5, count)
    thr = np.asarray(list(p.threshold))
    power = (thr[levels] * rng.uniform(0.9, 3.0, count)).astype(np.float32)
    c = np.zeros(count, B.CANDIDATE)
    c["bin"], c["level"], c["power"] = bins, levels, power
    order = np.lexsort((c["bin"], c["level"]))
    return c[order]


def test_toplist_matches_oracle_and_reference(oracle):
    rng = np.random.default_rng(11)
    p = B.search_parameters(1 << 20, 1 << 20, 128.0, 3600.0, 0.5, 0.1, 400.0, 0.08, 1000)
    tops = [B.Toplist(), oracle.Toplist()]
    if oracle.ref_available():
        tops.append(oracle.RefToplist())
    for t in range(300):
        c = _random_candidates(rng, p, int(rng.integers(0, 40)))
        # duplicate bins and exactly equal powers exercise the qsort tie order
        if t % 7 == 0 and len(c) > 2:
            c["power"][1] = c["power"][0]
            c["bin"][2] = c["bin"][0]
        orb = (3600.0 + t, 0.01 * t, 0.1 * t)
        for tl in tops:
            q = tl.thresholds(p)
            tl.retain(c, *orb, q)
        qs = [bytes(tl.thresholds(p)) for tl in tops]
        assert all(q == qs[0] for q in qs)
    finals = [tl.final() for tl in tops]
    for f in finals[1:]:
        assert f.tobytes() == finals[0].tobytes()
    assert len(finals[0]) > 0


def test_toplist_rejects_invalid_candidate():
    p = B.search_parameters(1 << 20, 1 << 20, 128.0, 3600.0, 0.5, 0.1, 400.0, 0.08, 1000)
    t = B.Toplist()
    c = np.zeros(1, B.CANDIDATE)
    c["bin"], c["level"], c["power"] = p.fundamental, 0, 100.0
    with pytest.raises(B.BrpError):
        t.retain(c, 1.0, 0.0, 0.0, p)


def test_toplist_fold_equals_sequential_retain(oracle):
    rng = np.random.default_rng(12)
    p = B.search_parameters(1 << 20, 1 << 20, 128.0, 3600.0, 0.5, 0.1, 400.0, 0.08, 1000)
    temps, orbs, cands = [], [], []
    for t in range(200):
        q = p.copy()
        for h in range(5):
            q.threshold[h] = p.threshold[h] * float(rng.uniform(0.95, 1.05))
        temps.append(q)
        orbs.append((3600.0 + t, 0.01 * t, 0.1 * t))
        cands.append(_random_candidates(rng, q, int(rng.integers(0, 25))))
    a = B.Toplist().fold(temps, orbs, cands).final()
    ref = oracle.Toplist()
    for q, o, c in zip(temps, orbs, cands):
        ref.retain(c, *o, ref.thresholds(q))
    assert a.tobytes() == ref.final().tobytes() and len(a) > 0


@pytest.mark.parametrize("quantum", [0.0, 0.5])
def test_toplist_long_stream_with_and_without_ties(oracle, quantum):
    """A long candidate stream (every template above the current row 100, as at
    the start of a bank) through the product's toplist, the oracle's and the
    reference's own code.  quantum > 0 rounds the powers so that many filled
    rows tie (the qsort path); quantum 0 keeps them distinct (the insertion path)."""
    rng = np.random.default_rng(13)
    p = B.search_parameters(1 << 20, 1 << 20, 128.0, 3600.0, 0.5, 0.1, 400.0, 0.08, 1000)
    tops = [B.Toplist(), oracle.Toplist()]
    if oracle.ref_available():
        tops.append(oracle.RefToplist())
    for t in range(150):
        c = _random_candidates(rng, p, 120)
        if quantum:
            c["power"] = np.round(c["power"] / quantum) * quantum
        orb = (3600.0 + t, 0.01 * t, 0.1 * t)
        for tl in tops:
            tl.retain(c, *orb, tl.thresholds(p))
    finals = [tl.final() for tl in tops]
    for f in finals[1:]:
        assert f.tobytes() == finals[0].tobytes()
    assert len(finals[0]) > 0


@pytest.mark.parametrize("shards", [1, 2, 3])
def test_toplist_prefilter_rule_keeps_the_final_rows(oracle, shards):
    """The rule of the device toplist pre-filter (brp_cuda_bank_set_toplist_filter),
    restated on the CPU: dropping every candidate below V, the 100th highest
    per-bin maximum of its level over the candidates it sees, leaves the final
    toplist unchanged -- for streams with repeated bins across templates, ties
    at V and thresholds that vary per template.  With the bank split into
    contiguous template shards (one per GPU) each shard takes its own V, which
    is at most the whole bank's, and the ranks' kept lists folded in bank order
    still give the same toplist."""
    rng = np.random.default_rng(21)
    p = B.search_parameters(1 << 20, 1 << 20, 128.0, 3600.0, 0.5, 0.1, 400.0, 0.08, 1000)
    temps, orbs, cands = [], [], []
    for t in range(120):
        q = p.copy()
        for h in range(5):
            q.threshold[h] = p.threshold[h] * float(rng.uniform(0.9, 1.1))
        c = _random_candidates(rng, q, 150)
        c["bin"] = p.window + rng.integers(0, 400, len(c))  # few distinct bins: many repeats
        c["power"] = np.round(c["power"] * 4) / 4            # ties, also at V
        keep = c["power"] > np.asarray(list(q.threshold))[c["level"]]
        c = c[keep]
        _, first = np.unique(np.stack([c["level"], c["bin"]]), axis=1, return_index=True)
        c = c[np.sort(first)]
        c = c[np.lexsort((c["bin"], c["level"]))]
        temps.append(q)
        orbs.append((3600.0 + t, 0.01 * t, 0.1 * t))
        cands.append(c)
    def threshold(lists):
        allc = np.concatenate(lists)
        V = np.zeros(5, np.float32)
        for h in range(5):
            lev = allc[allc["level"] == h]
            best = {}
            for b, pw in zip(lev["bin"].tolist(), lev["power"].tolist()):
                best[b] = max(best.get(b, -1.0), pw)
            maxima = sorted(best.values(), reverse=True)
            V[h] = maxima[99] if len(maxima) >= 100 else 0.0
        return V

    kept = []
    bounds = np.linspace(0, len(cands), shards + 1).astype(int)
    for a, b in zip(bounds[:-1], bounds[1:]):
        V = threshold(cands[a:b])
        kept += [c[c["power"] >= V[c["level"]]] for c in cands[a:b]]
    assert sum(map(len, kept)) < sum(map(len, cands)) // 2
    for make in (B.Toplist, oracle.Toplist):
        full, pre = make(), make()
        for q, o, c, k in zip(temps, orbs, cands, kept):
            full.retain(c, *o, full.thresholds(q))
            pre.retain(k, *o, pre.thresholds(q))
        assert full.final().tobytes() == pre.final().tobytes()
