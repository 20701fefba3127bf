"""Whitening and RFI zapping (src/workload.cpp:58-95) and DD decoding
(:29-57) on the CPU: the oracle's restatement against the reference's own
preprocess/load_observation compiled here (oracle/_ref, with the oracle's
stand-ins for FFTW, rngmed and GSL), the running median against its
definition, and the product's host zap-list reader and zap-noise generator
against the oracle."""

import numpy as np
import pytest

from brp_b200 import whiten
from dd_files import write_dd_bytes

N = 1 << 18
SAMPLE_US = 128.0


def series(samples, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(samples).astype(np.float32)
    t = np.arange(samples) * SAMPLE_US * 1e-6
    x += (0.3 * np.sin(2 * np.pi * 50.0 * t) + 0.2 * np.sin(2 * np.pi * 711.0 * t)).astype(np.float32)
    return x


def zap_file(tmp_path, rows, name="zap.txt"):
    p = tmp_path / name
    p.write_text("".join("%r %r\n" % r for r in rows))
    return p


def test_rngmed_matches_definition(oracle):
    rng = np.random.default_rng(1)
    x = rng.exponential(size=3000).astype(np.float32)
    x[100:140] = 2.0  # ties
    for w in (2, 8, 9, 100):
        got = oracle.rngmed(x, w)
        win = np.lib.stride_tricks.sliding_window_view(x, w)
        s = np.sort(win, axis=1)
        want = s[:, w // 2] if w % 2 else (np.float32(0.5) * (s[:, w // 2 - 1] + s[:, w // 2])).astype(np.float32)
        assert np.array_equal(got, want)


@pytest.mark.parametrize("n,samples,window", [(N, 200000, 1000), (3 << 16, 150000, 64)])
def test_oracle_preprocess_matches_reference(oracle, tmp_path, n, samples, window):
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    x = series(samples, 2)
    padding = n / samples
    seconds = n * SAMPLE_US * 1e-6
    rows = [(50.0 / seconds, 50.4 / seconds), (0.2, 0.2001)]
    zp = zap_file(tmp_path, rows)
    lo, hi = whiten.read_zap(zp)
    got = oracle.preprocess(x, n, SAMPLE_US, padding, window, lo, hi)
    ref = oracle.ref_preprocess(x, n, SAMPLE_US, padding, zp, window)
    assert np.array_equal(got, ref)
    assert np.all(np.isfinite(got)) and 0.5 < np.std(got) < 2.0


def test_zap_noise_product_equals_oracle(oracle):
    x0 = np.float32(0.123)
    seed = int(np.array([x0]).view(np.uint32)[0])
    lo, hi = np.array([0.1, 0.5, 0.3]), np.array([0.1005, 0.5002, 0.3001])
    bins, vals = whiten.zap_noise(seed, N, SAMPLE_US, 1.7, lo, hi)
    assert len(bins) > 0
    want = oracle.zap_noise(seed, len(bins), np.sqrt(2.0) / 2 * np.sqrt(1.7))
    assert np.array_equal(vals.reshape(-1), want)
    seconds = N * SAMPLE_US * 1e-6
    expect = np.concatenate([np.arange(int(l * seconds + 0.5), int(h * seconds + 0.5) + 1) for l, h in zip(lo, hi)])
    assert np.array_equal(bins, expect)
    # the restated generator is a Gaussian of the requested sigma
    g = oracle.zap_noise(7, 20000, 2.0)
    assert abs(g.mean()) < 0.05 and abs(g.std() - 2.0) < 0.05
    assert abs(np.mean(np.abs(g) > 2 * 2.0) - 0.0455) < 0.006


def test_zap_list_rules(tmp_path):
    lo, hi = whiten.read_zap(zap_file(tmp_path, [(0.1, 0.2), (0.3, 0.3)]))
    assert lo.tolist() == [0.1, 0.3] and hi.tolist() == [0.2, 0.3]
    for bad, msg in (("0.2 0.1\n", "invalid zap range"), ("0.1 0.2\n0.3\n", "malformed zap list"),
                     ("0.1 abc\n", "malformed zap list"), ("-1 0.5\n", "invalid zap range")):
        p = tmp_path / "bad.txt"
        p.write_text(bad)
        with pytest.raises(Exception, match=msg):
            whiten.read_zap(p)
    with pytest.raises(Exception, match="zap exceeds Nyquist"):
        whiten.zap_noise(1, N, SAMPLE_US, 1.0, [0.0], [1e9])


@pytest.mark.parametrize("packed", [False, True])
def test_dd_decode_matches_reference_loader(oracle, tmp_path, packed):
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    rng = np.random.default_rng(3)
    samples = 4096
    raw = rng.integers(0, 256, samples // 2 if packed else samples, dtype=np.uint8)
    path = tmp_path / ("obs.bin4" if packed else "obs.binary")
    write_dd_bytes(path, raw, samples, SAMPLE_US, scale=3.5)
    meta, ref = oracle.ref_load_observation(str(path), 1.0)
    assert meta[2] == samples
    assert np.array_equal(oracle.dd_decode(raw, samples, packed, 3.5), ref)
