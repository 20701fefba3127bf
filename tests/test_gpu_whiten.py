"""Whitening and RFI zapping on the GPU (brp_cuda_preprocess, _dd) against the
CPU oracle (oracle_preprocess, itself equal bit for bit to the reference's own
preprocess with the same FFT/median/RNG stand-ins): relative L2 of the
preprocessed series within 2e-6 (the reference's own gate against the authentic
application is 1e-4, src/workunit_main.cpp:62); zapped bins carry the same
noise; DD samples decoded on the device bit-exactly; the reference's errors."""
import os

import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import whiten

pytestmark = pytest.mark.gpu
SAMPLE_US = 128.0
REL_L2 = 2e-6


def series(samples, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(samples).astype(np.float32)
    t = np.arange(samples) * SAMPLE_US * 1e-6
    x += (0.3 * np.sin(2 * np.pi * 50.0 * t) + 0.2 * np.sin(2 * np.pi * 711.0 * t)).astype(np.float32)
    return x


def rel_l2(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n,samples,window", [(1 << 20, 900000, 1000), (3 << 18, 700000, 200), (1 << 16, 65536, 4096)])
def test_preprocess_matches_oracle(oracle, n, samples, window):
    x = series(samples, 5)
    padding = n / samples
    # zap ranges in the reference's units (Hz: bin = value * observation seconds + 0.5)
    lo, hi = np.array([49.9, 710.8, 1200.0]), np.array([50.2, 711.3, 1200.0])
    got = whiten.preprocess(x, n, SAMPLE_US, padding, window, (lo, hi))
    want = oracle.preprocess(x, n, SAMPLE_US, padding, window, lo, hi)
    err = rel_l2(got, want)
    print("n=%d window=%d: preprocessed relative L2 vs oracle %.3g" % (n, window, err))
    assert err <= REL_L2


def test_overlapping_zap_ranges_take_the_last_draw(oracle):
    n, samples = 1 << 18, 250000
    x = series(samples, 6)
    lo, hi = np.array([100.0, 100.2, 300.0]), np.array([100.4, 100.6, 300.1])  # the first two overlap
    got = whiten.preprocess(x, n, SAMPLE_US, n / samples, 1000, (lo, hi))
    want = oracle.preprocess(x, n, SAMPLE_US, n / samples, 1000, lo, hi)
    assert rel_l2(got, want) <= REL_L2


def test_dd_decoding_on_the_device(oracle):
    rng = np.random.default_rng(9)
    n, samples = 1 << 18, 240000
    for packed in (False, True):
        raw = rng.integers(0, 256, samples // 2 if packed else samples, dtype=np.uint8)
        dec, out = whiten.preprocess_dd(raw, samples, packed, 2.5, n, SAMPLE_US, n / samples, 1000)
        assert np.array_equal(dec, oracle.dd_decode(raw, samples, packed, 2.5))
        again = whiten.preprocess(dec, n, SAMPLE_US, n / samples, 1000)
        assert np.array_equal(out, again)
        assert rel_l2(out, oracle.preprocess(dec, n, SAMPLE_US, n / samples, 1000)) <= REL_L2


def test_preprocess_errors():
    x = series(60000, 1)
    n = 1 << 16
    for window, msg in ((999, "unsupported whitening window"), (8192, "4096")):
        with pytest.raises(B.BrpError, match=msg):
            whiten.preprocess(x, n, SAMPLE_US, n / 60000, window)
    with pytest.raises(B.BrpError, match="zap exceeds Nyquist"):
        whiten.preprocess(x, n, SAMPLE_US, n / 60000, 1000, ([0.0], [1e9]))
    with pytest.raises(B.BrpError, match="invalid whitening median"):
        whiten.preprocess(np.zeros(60000, np.float32), n, SAMPLE_US, n / 60000, 1000)


def test_against_reference_golden():
    """The device whitening against the reference's own preprocess output
    (tests/golden/whitening_vectors.npz, made by src/workload.cpp compiled with
    the oracle's stand-ins) within the same relative L2 bar, and the device DD
    decoding bit-exact against the reference loader's samples."""
    W = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "whitening_vectors.npz"))
    for k in (0, 1):
        n, samples, window, padding = W["pre_case_%d" % k]
        rows = W["pre_zap_%d" % k]
        got = whiten.preprocess(W["pre_input_%d" % k], int(n), SAMPLE_US, float(padding), int(window),
                                (rows[:, 0], rows[:, 1]))
        err = rel_l2(got, W["pre_output_%d" % k])
        print("golden case %d (n=%d): preprocessed relative L2 vs the reference %.3g" % (k, int(n), err))
        assert err <= REL_L2
    for name, packed in (("int8", False), ("packed", True)):
        sample_us, scale, samples, _ = W["dd_meta_" + name]
        n = 8192  # the device whitening's shortest length
        dec, _ = whiten.preprocess_dd(W["dd_raw_" + name], int(samples), packed, float(scale), n, float(sample_us),
                                      n / samples, 1000)
        assert np.array_equal(dec.view(np.uint32), W["dd_decoded_" + name].view(np.uint32))
