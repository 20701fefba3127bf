"""The oracle against the reference's own compiled CPU code (oracle/_ref) on
seeded random templates (CPU).

The golden vectors pin the oracle on a fixed set of cases; here the oracle's
template constants (src/science.cpp:46-65), resampling steps, production
(FMA) constants and resampled series (src/science.cpp:75-85, both
arithmetics) are compared bit for bit with the reference's compiled functions
on random orbits, lengths, paddings and sample times, and the search
parameters (src/workload.cpp:108-125) on random observations.  Where one side
rejects its arguments the other must reject them too.  Skipped where the
reference build is absent.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference build absent (oracle/_ref)")

LENGTHS = [1 << 13, 3 << 12, 1 << 14, 3 << 13, 1 << 15, 1 << 16]
DTS = [1e-3, 2.56e-4, 6.4e-5]


def both(fo, fr):
    """(oracle result, reference result), or (None, None) when both reject."""
    try:
        a = fo()
    except O.OracleError:
        a = None
    try:
        b = fr()
    except O.OracleError:
        b = None
    assert (a is None) == (b is None), "one side rejected the arguments"
    return a, b


def ref_production(p):
    """The production constants as the reference's driver forms them (src/main.cpp:41)."""
    q = O.Params.from_buffer_copy(bytes(p))
    q.flags = 2 | 4
    q.s0 = np.float32(np.float32(q.tau) * np.float32(np.sin(np.float32(q.psi)))) * np.float32(q.step_inv)
    return O.ref_resampling_steps(q)


@pytest.mark.parametrize("seed", range(8))
def test_constants_and_resampling_match_the_reference(oracle, seed):
    rng = np.random.default_rng(1000 + seed)
    for _ in range(6):
        n = int(rng.choice(LENGTHS))
        unpadded = n - int(rng.integers(0, 65))
        tau = float(rng.uniform(0.0, 3.2))
        period = float(rng.uniform(300.0, 30000.0))
        psi = float(rng.uniform(-7.0, 7.0))
        dt = float(rng.choice(DTS))
        po, pr = both(lambda: oracle.parameters(n, unpadded, tau, period, psi, dt),
                      lambda: oracle.ref_parameters(n, unpadded, tau, period, psi, dt))
        if po is None:
            continue
        assert bytes(po) == bytes(pr)
        x = rng.standard_normal(unpadded).astype(np.float32)
        ro, rr = oracle.resample(x, po), oracle.ref_resample(x, pr)
        assert np.array_equal(ro[:po.steps].view(np.uint32), rr[:pr.steps].view(np.uint32))
        qo, qr = both(lambda: oracle.production(po), lambda: ref_production(pr))
        if qo is None:
            continue
        assert bytes(qo) == bytes(qr)
        ro, rr = oracle.resample(x, qo), oracle.ref_resample(x, qr)
        assert np.array_equal(ro[:qo.steps].view(np.uint32), rr[:qr.steps].view(np.uint32))


@pytest.mark.parametrize("seed", range(4))
def test_search_parameters_match_the_reference(oracle, seed):
    rng = np.random.default_rng(2000 + seed)
    for _ in range(10):
        n = int(rng.choice([1 << 16, 3 << 15, 1 << 18, 1 << 20, 1 << 22]))
        samples = n - int(rng.integers(0, n // 8))
        sample_us = float(rng.choice([64.0, 128.0, 256.0, 500.0]))
        period = float(rng.uniform(600.0, 40000.0))
        tau = float(rng.uniform(0.0, 3.0))
        psi = float(rng.uniform(0.0, 2 * np.pi))
        f0 = float(rng.choice([200.0, 400.0, 800.0]))
        fa = float(rng.choice([0.01, 0.08, 0.5]))
        window = int(rng.choice([100, 500, 1000]))
        po, pr = both(lambda: oracle.search_parameters(n, samples, sample_us, period, tau, psi, f0, fa, window),
                      lambda: oracle.ref_search_parameters(n, samples, sample_us, period, tau, psi, f0, fa, window))
        if po is not None:
            assert bytes(po) == bytes(pr)


@pytest.mark.parametrize("seed", range(6))
def test_pipeline_matches_the_reference(oracle, seed):
    """The whole CPU path (src/science.cpp:113-120) of the reference's compiled
    code, with its FFTW stand-in (the FP64 DFT rounded to float), against the
    oracle's resampling, the same DFT, power, harmonic sums and selection, on a
    random template over a series with an injected pulsar; the thresholds are
    lowered to a high quantile of each level so that every level selects.  The
    reference build's harmonic step is the stand-in for the absent hs_common.c
    (the same restatement as the oracle's), so the harmonic sums are not an
    independent check; resampling, power and selection are."""
    from brp_b200 import synth
    rng = np.random.default_rng(3000 + seed)
    n = int(rng.choice([1 << 12, 3 << 11, 1 << 13, 3 << 12, 1 << 14]))
    unpadded = n - int(rng.integers(1, 40))
    pul = synth.Pulsar(float(rng.uniform(50.0, 900.0)), float(rng.uniform(600.0, 20000.0)),
                       float(rng.uniform(0.0, 1.5)), float(rng.uniform(0.0, 6.2)), 0.3, 5, 0.1)
    x = synth.make_series(unpadded, seed, [pul])
    p = oracle.ref_parameters(n, unpadded, pul.tau, pul.period, pul.psi, synth.DT)
    if seed % 2:
        p = ref_production(p)
    ref = oracle.ref_reference(x, p)
    q = O.Params.from_buffer_copy(bytes(p))
    for h in range(5):  # the same lowered thresholds on both sides
        lvl = ref["summed"][h * p.fundamental:(h + 1) * p.fundamental]
        q.threshold[h] = float(np.float32(np.quantile(lvl[p.window:], 0.995)))
    ref = oracle.ref_reference(x, q)
    r = oracle.resample(x, q)
    assert np.array_equal(r.view(np.uint32), ref["resampled"].view(np.uint32))
    X = oracle.rfft64_c(r)
    Xf = X.real.astype(np.float32) + 1j * X.imag.astype(np.float32)
    P = oracle.power_from_fft(Xf.astype(np.complex128), q.n)
    assert np.array_equal(P.view(np.uint32), ref["power"].view(np.uint32))
    S = oracle.harmonic(P, q)
    assert np.array_equal(S.view(np.uint32), ref["summed"].view(np.uint32))
    c = oracle.select(S, q)
    assert len(c) > 0 and set(int(v) for v in c["level"]) == set(range(5))
    assert c.tobytes() == ref["candidates"].tobytes()
