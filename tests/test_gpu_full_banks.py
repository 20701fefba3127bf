"""The benchmark banks at full size against the CPU oracle (slow).

* The N = 2^22 bank of 512 templates with 3 injected pulsars (the bench
  workload, toplist pre-filter off): every template's candidate list against
  the oracle pipeline (the reference's resampling, an FP64 FFT, the restated
  harmonic sum and select), identical except within 1e-5 relative of a
  threshold; the bank-wide toplist folded from the GPU's lists equal to the
  one folded from the oracle's, row for row.
* The mixed-radix bank (N = 3*2^21, 128 templates, 2 pulsars) in the FP32
  CUDA-core form: the same per-template and toplist checks, plus the first
  template's power against an FP64 FFT of its own padded series, and its
  harmonic sums and candidates bit-exact against the restated shader fed the
  GPU's power.  The tensor-core forms of pass 1 are compared with the oracle
  too: their candidate differences must all lie near a threshold.
The oracle runs in a pool of host processes; the gates mirror the
reference's own (src/main.cpp:55-80, src/workunit_main.cpp:103-122)."""
import multiprocessing as mp
import os

import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import shard, synth

pytestmark = [pytest.mark.gpu, pytest.mark.slow]
POWER_RTOL = 2e-6
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
    return O.pipeline(_W["series"][s], O.Params.from_buffer_copy(pbytes))["candidates"]


def oracle_lists(wl):
    ctx = mp.get_context("spawn")
    with ctx.Pool(max(2, min(32, os.cpu_count() or 2)), initializer=_init, initargs=(wl.series,)) as pool:
        return pool.map(_oracle_candidates, [(int(s), bytes(p)) for s, p in zip(wl.series_of, wl.templates)],
                        chunksize=2)


def differences(got, ref, p, rtol):
    """(keys in one list only, keys in one list only that are not within rtol of
    their threshold, largest relative power difference of the shared keys)."""
    kg = {(int(b), int(l)): float(v) for b, l, v in zip(got["bin"], got["level"], got["power"])}
    kr = {(int(b), int(l)): float(v) for b, l, v in zip(ref["bin"], ref["level"], ref["power"])}
    only = set(kg) ^ set(kr)
    far = [k for k in only
           if abs(kg.get(k, kr.get(k)) - float(p.threshold[k[1]])) > rtol * float(p.threshold[k[1]])]
    worst = max([abs(kg[k] - kr[k]) / max(abs(kr[k]), 1e-30) for k in set(kg) & set(kr)] or [0.0])
    return len(only), len(far), worst


def run_bank(wl, **configure):
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    for s, x in enumerate(wl.series):
        bank.set_series(s, x)
    if configure:
        bank.configure(wl.n[0], **configure)
    got, counts, status = bank.run(wl.templates, wl.series_of)
    bank.close()
    assert not status.any()
    return got


def assert_bank_matches(wl, got, ref, rtol=1e-5):
    only = far = 0
    worst = 0.0
    for g, r, p in zip(got, ref, wl.templates):
        a, b, w = differences(g, r, p, rtol)
        only, far, worst = only + a, far + b, max(worst, w)
    total = sum(len(c) for c in got)
    print("%s: %d GPU candidates, %d oracle, %d differ (%d away from a threshold), largest shared power "
          "difference %.3g" % (wl.name, total, sum(len(c) for c in ref), only, far, worst))
    assert total > 100 and far == 0 and worst <= 2e-4
    top = shard.fold_toplist(B.Toplist(), wl.templates, wl.orbits, got).final()
    rtop = shard.fold_toplist(B.Toplist(), wl.templates, wl.orbits, ref).final()
    assert len(top) == len(rtop) == 100
    for x, y in zip(top, rtop):
        assert (x["bin"], x["harmonics"], x["period"], x["tau"], x["psi"]) == \
               (y["bin"], y["harmonics"], y["period"], y["tau"], y["psi"])


def test_bench_bank_512_templates_n2e22():
    wl = synth.config3(512)
    assert_bank_matches(wl, run_bank(wl), oracle_lists(wl))


@pytest.fixture(scope="module")
def mixed_radix():
    wl = synth.config4(128)
    return wl, oracle_lists(wl)


def test_mixed_radix_bank_fp32(oracle, mixed_radix):
    wl, ref = mixed_radix
    got = run_bank(wl)  # the default (tuned) FP32 plan: pass 1 = 119, pass 2 = 207
    assert_bank_matches(wl, got, ref)
    p = wl.templates[0]
    g = B.GPU(p, wl.series[0], 256, 0, 1, stockham=True, packed=True)
    g.set_template(p)
    g.run()
    s = g.snapshot()
    g.close()
    P64 = oracle.power64(oracle.rfft64(s.resampled), p.n)
    err = float(np.sqrt(np.sum((s.power - P64) ** 2) / np.sum(P64 ** 2)))
    assert err <= POWER_RTOL
    assert np.array_equal(s.summed, oracle.harmonic(s.power, p))
    assert np.array_equal(s.candidates, oracle.select(s.summed, p))
    assert np.array_equal(s.candidates, got[0])


@pytest.mark.parametrize("pass1,terms", [(113, 3), (114, 2)])
def test_mixed_radix_bank_tensor_cores_vs_oracle(mixed_radix, pass1, terms):
    wl, ref = mixed_radix
    got = run_bank(wl, pass1=pass1, pass2=0, group=16, chains=2)
    only = far = 0
    for g, r, p in zip(got, ref, wl.templates):
        a, b, _ = differences(g, r, p, 1e-5 if terms == 3 else 1e-4)
        only, far = only + a, far + b
    print("bank n=3*2^21: pass1 %d (%d BF16 parts): %d of %d candidates differ from the oracle, %d away from a "
          "threshold" % (pass1, terms, only, sum(len(c) for c in ref), far))
    assert far == 0
