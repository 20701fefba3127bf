"""Tensor-core form of pass 1 (compiled pass-1 configurations 111-114: the
first radix-16 stage of the column FFTs as split-BF16 DFT products on the
tensor cores, FP32 accumulation) against the FP64 FFT oracle and against the
FP32 CUDA-core form of the same decomposition (110 for n = 2^22, 119 for
n = 3*2^21).

Three BF16 parts per operand (111, 113) carry every bit of an FP32 operand and
are held to the CUDA-core bars: power within 2e-6 relative RMS of FP64,
candidates identical except within 1e-5 relative of a threshold.  The hi/lo
split (112, 114) carries 16 bits per operand; its power error is reported and
bounded at 2e-5, and its candidate lists may differ from the FP32 form only
near a threshold (within 1e-4 relative).  Each case prints its measured error
and the candidate differences."""
import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import synth

pytestmark = pytest.mark.gpu
POWER_RTOL = {3: 2e-6, 2: 2e-5}
THRESH_RTOL = {3: 1e-5, 2: 1e-4}
# tensor-core id: (CUDA-core id of the same radix sequence, n, BF16 parts)
TC = {111: (110, 1 << 22, 3), 112: (110, 1 << 22, 2), 113: (119, 3 << 21, 3), 114: (119, 3 << 21, 2)}


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def run_gpu(p, x, pass1):
    g = B.GPU(p, x, 192, 0, 1, stockham=True, packed=True, pass1=pass1)
    g.set_template(p)
    g.run()
    s = g.snapshot()
    g.close()
    return s


def candidate_differences(got, ref, p, rtol):
    """(number of (bin, level) keys in only one list, all of them within rtol of a threshold)."""
    kg = {(int(b), int(l)): float(v) for b, l, v in zip(got["bin"], got["level"], got["power"])}
    kr = {(int(b), int(l)): float(v) for b, l, v in zip(ref["bin"], ref["level"], ref["power"])}
    diff = set(kg) ^ set(kr)
    near = all(abs(kg.get(k, kr.get(k)) - float(p.threshold[k[1]])) <= rtol * float(p.threshold[k[1]])
               for k in diff)
    return len(diff), near


@pytest.mark.parametrize("tc", sorted(TC))
def test_tensor_form_vs_fp64_and_cuda_cores(oracle, tc):
    base, n, terms = TC[tc]
    unp = n - 17
    pul = synth.Pulsar(421.3, 11 * 3600.0, 1.7, 0.4, 0.01, 8, 0.1)
    x = synth.make_series(unp, 9, [pul])
    p = B.production(B.parameters(n, unp, pul.tau, pul.period, pul.psi, synth.DT))
    s = run_gpu(p, x, tc)
    r = run_gpu(p, x, base)
    # the resampling is shared with the CUDA-core form: bit-exact
    assert np.array_equal(s.resampled[:p.steps], oracle.resample(x, p)[:p.steps])
    P64 = oracle.power64(oracle.rfft64(s.resampled), n)
    err_tc, err_fp32 = rel_rms(s.power, P64), rel_rms(r.power, P64)
    assert err_tc <= POWER_RTOL[terms]
    # harmonic sums of the tensor-core power are those of the restated shader
    assert np.array_equal(s.summed, oracle.harmonic(s.power, p))
    ndiff, near = candidate_differences(s.candidates, r.candidates, p, THRESH_RTOL[terms])
    print("pass1 %d (%d BF16 parts) n=%d: power rel RMS vs FP64 %.3g (FP32 form %.3g); candidates %d vs %d, "
          "%d differ" % (tc, terms, n, err_tc, err_fp32, len(s.candidates), len(r.candidates), ndiff))
    assert near
    assert len(r.candidates) > 0


def test_tensor_form_bank_mixed_radix():
    """The mixed-radix bank (n = 3*2^21, 2 pulsars, 128 templates) with pass 1 in
    the tensor-core form against the same bank in the FP32 CUDA-core form."""
    wl = synth.config4()
    n = wl.n[0]
    lists = {}
    for p1 in (119, 113, 114):
        bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
        bank.set_series(0, wl.series[0])
        bank.configure(n, pass1=p1, pass2=0, group=16, chains=2)
        got, counts, status = bank.run(wl.templates, wl.series_of)
        assert not status.any()
        lists[p1] = got
        bank.close()
    total = sum(len(c) for c in lists[119])
    assert total > 0
    for p1, terms in ((113, 3), (114, 2)):
        ndiff = 0
        for g, r, p in zip(lists[p1], lists[119], wl.templates):
            d, near = candidate_differences(g, r, p, THRESH_RTOL[terms])
            assert near
            ndiff += d
        print("bank n=3*2^21, 128 templates: pass1 %d (%d BF16 parts) %d of %d candidates differ from the FP32 form"
              % (p1, terms, ndiff, total))
