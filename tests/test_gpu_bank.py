"""Bank search (one captured CUDA graph over templates of several series
lengths) against the CPU oracle run template by template, and the bank-wide
toplist against the oracle's toplist (src/workload.cpp:126-159)."""
import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import shard, synth

pytestmark = pytest.mark.gpu
THRESH_RTOL = 1e-5


def cand_map(c):
    return {(int(b), int(l)): float(v) for b, l, v in zip(c["bin"], c["level"], c["power"])}


def assert_same_candidates(got, ref, p):
    kg, kr = cand_map(got), cand_map(ref)
    for k in set(kg) | set(kr):
        thr = float(p.threshold[k[1]])
        if k in kg and k in kr:
            assert abs(kg[k] - kr[k]) <= 2e-4 * (1 + abs(kr[k])), k
        else:
            v = kg.get(k, kr.get(k))
            assert abs(v - thr) <= THRESH_RTOL * thr, (k, v, thr)


def oracle_bank(oracle, wl):
    out = []
    for p, s in zip(wl.templates, wl.series_of):
        out.append(oracle.pipeline(wl.series[s], p)["candidates"])
    return out


@pytest.fixture(scope="module")
def small_bank():
    # three lengths (2^16, 3*2^15, 2^17), uneven counts, pulsars strong enough
    # for candidates at 5 and 7 sigma thresholds
    return synth.bank_workload("small-uneven", [1 << 16, 3 << 15, 1 << 17], [9, 5, 3], [2, 1, 1], seed=21,
                               f0=800.0, sigmas=(5.0, 7.0))


def test_bank_matches_oracle(oracle, small_bank):
    wl = small_bank
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    for s, x in enumerate(wl.series):
        bank.set_series(s, x)
    got, counts, status = bank.run(wl.templates, wl.series_of)
    assert not status.any()
    ref = oracle_bank(oracle, wl)
    total = 0
    for g, r, p in zip(got, ref, wl.templates):
        assert_same_candidates(g, r, p)
        total += len(g)
    assert total > 0
    # replay: the same graph again gives identical results
    got2, _, _ = bank.run(wl.templates, wl.series_of)
    for a, b in zip(got, got2):
        assert np.array_equal(a, b)
    bank.close()


def test_bank_matches_single_template_path(small_bank):
    wl = small_bank
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    for s, x in enumerate(wl.series):
        bank.set_series(s, x)
    got, _, _ = bank.run(wl.templates, wl.series_of)
    for t in (0, 9, 14):
        p, s = wl.templates[t], wl.series_of[t]
        g = B.GPU(p, wl.series[s], 256, 0, 1, stockham=True, packed=True)
        g.set_template(p)
        g.run()
        assert np.array_equal(g.candidates(), got[t])
        g.close()
    bank.close()


def test_bank_toplist_equals_oracle(oracle, small_bank):
    wl = small_bank
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    for s, x in enumerate(wl.series):
        bank.set_series(s, x)
    got, _, _ = bank.run(wl.templates, wl.series_of)
    top = shard.fold_toplist(B.Toplist(), wl.templates, wl.orbits, got).final()
    ref_top = shard.fold_toplist(oracle.Toplist(), wl.templates, wl.orbits, oracle_bank(oracle, wl)).final()
    assert len(top) == len(ref_top) and len(top) > 0
    for a, b in zip(top, ref_top):
        assert (a["bin"], a["harmonics"], a["period"], a["tau"], a["psi"]) == \
               (b["bin"], b["harmonics"], b["period"], b["tau"], b["psi"])
        assert abs(a["power"] - b["power"]) <= 2e-5 * abs(b["power"])
    bank.close()


def test_bank_overflow_reported():
    wl = synth.bank_workload("overflow", [1 << 16], [2], [1], seed=5, f0=800.0, sigmas=(5.0,))
    t = [p.copy() for p in wl.templates]
    for p in t:
        for h in range(5):
            p.threshold[h] = 0.0  # every bin qualifies
    bank = B.Bank(wl.n, [len(wl.series[0])], 2, 64)
    bank.set_series(0, wl.series[0])
    with pytest.raises(B.BrpError) as e:
        bank.run(t)
    assert (e.value.status & B.STATUS_OVERFLOW).all()
    bank.close()


def test_resample_out_of_range_reported():
    n = 1 << 16
    x = synth.make_series(n, 1)
    p = B.search_parameters(n, n, 128.0, 3600.0, 0.5, 1.0, 400.0, 0.08, 1000)
    bad = p.copy()
    bad.s0 = -3000.0  # offset(i) grows by 3000 samples: the first indices fall before the series
    bank = B.Bank([n], [n], 1, 1024)
    bank.set_series(0, x)
    with pytest.raises(B.BrpError) as e:
        bank.run([bad])
    assert e.value.status[0] & B.STATUS_RESAMPLE_OOB
    bank.close()


def test_configure_drops_the_graph_and_frees_replaced_buffers():
    """brp_cuda_bank_configure drops the captured graph (a replay before the
    next run is refused instead of reading replaced plan tables) and frees the
    class buffers it replaces when a larger group needs more: growing a 2^20
    class (6 MiB of intermediates per template) from 64 to 128 templates costs
    the difference, not a second full set."""
    import torch
    wl = synth.bank_workload("configure", [1 << 20], [64], [1], seed=8)
    bank = B.Bank(wl.n, [len(x) for x in wl.series], 64, 8192)
    bank.set_series(0, wl.series[0])
    first, _, _ = bank.run(wl.templates)
    bank.launch()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    bank.configure(1 << 20, pass1=0, pass2=0, group=64, chains=2)  # 128 templates' buffers
    free1 = torch.cuda.mem_get_info()[0]
    with pytest.raises(B.BrpError, match="no captured bank graph"):
        bank.launch()
    again, _, _ = bank.run(wl.templates)
    bank.launch()
    torch.cuda.synchronize()
    bank.close()
    grown = (free0 - free1) / (1 << 20)
    print("configure 64 -> 2 x 64 templates: %.0f MiB more device memory" % grown)
    assert 300 <= grown <= 500  # 64 x 6 MiB = 384 MiB (not 768)
    for a, b in zip(first, again):
        assert np.array_equal(a, b)


def test_submit_wait_with_an_upload_in_flight(small_bank):
    """brp_cuda_bank_submit / brp_cuda_bank_wait: a series uploaded while a run
    is in flight goes to the other buffer, so that run still searches the old
    series and the next one the new; calls that touch the bank's buffers are
    refused until the wait."""
    wl = small_bank
    other = [x[::-1].copy() for x in wl.series]  # a different series of the same lengths

    def fresh(series):
        bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
        for s, x in enumerate(series):
            bank.set_series(s, x)
        return bank

    ref_bank = fresh(wl.series)
    ref_old, _, _ = ref_bank.run(wl.templates, wl.series_of)
    ref_bank.close()
    ref_bank = fresh(other)
    ref_new, _, _ = ref_bank.run(wl.templates, wl.series_of)
    ref_bank.close()

    bank = fresh(wl.series)
    bank.submit(wl.templates, wl.series_of)
    for s, x in enumerate(other):
        bank.set_series(s, x)  # while the run is in flight
    with pytest.raises(B.BrpError) as e:
        bank.configure(wl.n[0], group=4)
    assert e.value.status == 4
    with pytest.raises(B.BrpError):
        bank.submit(wl.templates, wl.series_of)
    flat, offs, counts, status = bank.wait()
    assert not status.any()
    for t, r in enumerate(ref_old):
        assert np.array_equal(flat[offs[t]:offs[t + 1]], r)
    got, _, _ = bank.run(wl.templates, wl.series_of)
    for a, b in zip(got, ref_new):
        assert np.array_equal(a, b)
    with pytest.raises(B.BrpError):
        bank.wait()
    bank.close()
