"""The CPU oracle and the product's host code against golden vectors produced
by the reference's own CPU code (tests/golden/make_golden.py, from
src/science.cpp and src/workload.cpp compiled unmodified).  Bit-exact."""
import os

import numpy as np
import pytest

import brp_b200 as B

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.npz")


@pytest.fixture(scope="module")
def G():
    return np.load(GOLDEN)


def as_params(O, raw):
    return O.Params.from_buffer_copy(raw.tobytes())


def test_lut_sin(oracle, G):
    got = np.array([oracle.lut_sin(x) for x in G["lut_x"]], np.float32)
    assert np.array_equal(got.view(np.uint32), G["lut_sin"].view(np.uint32))


def test_parameters_and_indices(oracle, G):
    for k, c in enumerate(G["param_cases"]):
        n, unp = int(c[0]), int(c[1])
        p = oracle.parameters(n, unp, *c[2:])
        assert bytes(p) == G["params"][k].tobytes()
        assert bytes(B.parameters(n, unp, *c[2:])) == G["params"][k].tobytes()
        q = oracle.production(p)
        assert bytes(q) == G["params_production"][k].tobytes()
        assert bytes(B.production(B.parameters(n, unp, *c[2:]))) == G["params_production"][k].tobytes()
        x = np.arange(p.unpadded, dtype=np.float32)
        _, idx = oracle.resample(x, p, with_index=True)
        assert np.array_equal(idx, G["index_%d" % k])
        _, idx = oracle.resample(x, q, with_index=True)
        assert np.array_equal(idx, G["index_production_%d" % k])


def test_search_parameters(oracle, G):
    for k, c in enumerate(G["search_cases"]):
        args = (int(c[0]), int(c[1]), *c[2:8], int(c[8]))
        assert bytes(oracle.search_parameters(*args)) == G["search_params"][k].tobytes()
        assert bytes(B.search_parameters(*args)) == G["search_params"][k].tobytes()


def test_harmonic_sums(oracle, G):
    for k in range(4):
        p = as_params(oracle, G["hs_params_%d" % k])
        S = oracle.harmonic(G["hs_power_%d" % k], p)
        assert np.array_equal(S, G["hs_summed_%d" % k])


def test_reference_pipeline(oracle, G):
    p = as_params(oracle, G["pipe_params"])
    x = G["pipe_input"]
    r, _ = oracle.resample(x, p, with_index=True)
    assert np.array_equal(r, G["pipe_resampled"])
    X = oracle.rfft64_c(r)  # the reference's FFTW is replaced by the same FP64 DFT
    Xf = X.real.astype(np.float32) + 1j * X.imag.astype(np.float32)
    P = oracle.power_from_fft(Xf.astype(np.complex128), p.n)
    assert np.array_equal(P, G["pipe_power"])
    S = oracle.harmonic(P, p)
    assert np.array_equal(S, G["pipe_summed"])
    c = oracle.select(S, p)
    assert c.tobytes() == G["pipe_candidates"].tobytes()
    assert len(c) > 0


@pytest.mark.parametrize("impl", ["oracle", "product"])
def test_toplist(oracle, G, impl):
    p = as_params(oracle, G["top_params"])
    tl = oracle.Toplist() if impl == "oracle" else B.Toplist()
    off = 0
    cands = G["top_cands"]
    for cnt, orb in zip(G["top_counts"], G["top_orbits"]):
        q = tl.thresholds(p)
        tl.retain(cands[off:off + cnt], *orb, q)
        off += cnt
    assert tl.final().tobytes() == G["top_final"].tobytes()


def test_fp64_dft_matches_numpy(oracle):
    rng = np.random.default_rng(3)
    for n in (64, 96, 3 * 1024, 1 << 14):
        x = rng.standard_normal(n).astype(np.float32)
        a, b = oracle.rfft64_c(x), oracle.rfft64(x)
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


def test_chisq_inverse_roundtrip(oracle):
    for nu in (2, 4, 8, 16, 32):
        for q in (0.5, 1e-3, 1e-8, 1e-14):
            x = oracle.chisq_Qinv(q, nu)
            assert abs(oracle.chisq_Q(x, nu) / q - 1) < 1e-12
    # closed form at nu = 2: Q = exp(-x/2)
    assert abs(oracle.chisq_Q(10.0, 2) - np.exp(-5.0)) < 1e-15


WHITENING = os.path.join(os.path.dirname(GOLDEN), "whitening_vectors.npz")


@pytest.fixture(scope="module")
def W():
    return np.load(WHITENING)


@pytest.mark.parametrize("k", [0, 1])
def test_whitening_golden(oracle, W, k):
    """brp::preprocess (src/workload.cpp:58-95) by the oracle against the
    reference's own output (tests/golden/make_whitening_golden.py); the zap
    rows go through the product's zap-list reader first."""
    import tempfile

    from brp_b200 import whiten
    n, samples, window, padding = W["pre_case_%d" % k]
    rows = W["pre_zap_%d" % k]
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "zap.txt")
        with open(path, "w") as f:
            f.write("".join("%r %r\n" % (float(a), float(b)) for a, b in rows))
        lo, hi = whiten.read_zap(path)
    assert np.array_equal(lo, rows[:, 0]) and np.array_equal(hi, rows[:, 1])
    got = oracle.preprocess(W["pre_input_%d" % k], int(n), 128.0, float(padding), int(window), lo, hi)
    assert np.array_equal(got.view(np.uint32), W["pre_output_%d" % k].view(np.uint32))


@pytest.mark.parametrize("name,packed", [("int8", False), ("packed", True)])
def test_dd_decoding_golden(oracle, W, name, packed):
    """DD sample decoding of brp::load_observation (src/workload.cpp:48-56):
    bit-exact, with the reference loader's sample count and scale."""
    sample_us, scale, samples, n = W["dd_meta_" + name]
    assert sample_us == 128.0 and scale == 3.5
    got = oracle.dd_decode(W["dd_raw_" + name], int(samples), packed, scale)
    assert np.array_equal(got.view(np.uint32), W["dd_decoded_" + name].view(np.uint32))
