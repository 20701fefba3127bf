"""brp_cuda_search_static: the search for callers that cannot allocate device
memory (it keeps its working memory in a static device array of the library).
Its power spectrum and candidates must agree with the regular entry point
(brp_cuda_create/run through brp_b200.GPU) within the parity tolerances of the
other GPU tests, on consecutive calls that reuse the same static array.

This file is collected last so that a run stopping at the first failure has
run every other test before it; it also passes when run on its own."""
import ctypes

import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import synth
from brp_b200._lib import as_params, lib

pytestmark = pytest.mark.gpu
POWER_RTOL = 2e-6
THRESH_RTOL = 1e-5


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def static_search(p, x, capacity=1 << 16):
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    d_x = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(dev)
    d_power = torch.empty(p.n // 2, dtype=torch.float32, device=dev)
    d_cands = torch.empty(capacity * 4, dtype=torch.int32, device=dev)
    d_count = torch.empty(1, dtype=torch.int32, device=dev)
    d_status = torch.empty(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    q = as_params(p)
    st = lib().brp_cuda_search_static(ctypes.byref(q), d_x.data_ptr(), d_power.data_ptr(), d_cands.data_ptr(),
                                      capacity, d_count.data_ptr(), d_status.data_ptr(), stream.cuda_stream)
    assert st == 0, lib().brp_cuda_search_static_error().decode()
    torch.cuda.synchronize(dev)
    count, status = int(d_count.item()), int(d_status.item())
    assert status == 0 and count <= capacity
    c = d_cands.cpu().numpy().view(B.CANDIDATE)[:count]
    c = c[np.lexsort((c["bin"], c["level"]))]
    return d_power.cpu().numpy(), c


def regular_search(p, x):
    g = B.GPU(p, x, 256, 0, 1, stockham=True, packed=True)
    g.set_template(p)
    g.run()
    s = g.snapshot()
    g.close()
    return s.power, s.candidates


def assert_same(got, ref, p):
    (pw, c), (pw_ref, c_ref) = got, ref
    assert rel_rms(pw, pw_ref) <= POWER_RTOL
    kg = {(int(b), int(l)): float(v) for b, l, v in zip(c["bin"], c["level"], c["power"])}
    kr = {(int(b), int(l)): float(v) for b, l, v in zip(c_ref["bin"], c_ref["level"], c_ref["power"])}
    for k in set(kg) | set(kr):
        thr = float(p.threshold[k[1]])
        if k in kg and k in kr:
            assert abs(kg[k] - kr[k]) <= 2e-4 * (1 + abs(kr[k])), k
        else:
            v = kg.get(k, kr.get(k))
            assert abs(v - thr) <= THRESH_RTOL * thr, (k, v, thr)


def test_static_search_matches_regular_entry_point(oracle):
    cases = [
        (1 << 20, synth.Pulsar(311.0, 9000.0, 1.3, 0.7, 0.02, 8, 0.1), 5, True),
        (1 << 20, synth.Pulsar(97.0, 5000.0, 0.4, 2.9, 0.03, 5, 0.1), 6, False),  # second call, same array
        (3 << 16, synth.Pulsar(211.0, 7200.0, 0.8, 2.0, 0.06, 8, 0.1), 7, True),  # new length: tables refilled
    ]
    found = 0
    for n, pul, seed, prod in cases:
        x = synth.make_series(n - 17, seed, [pul])
        p = B.parameters(n, n - 17, pul.tau, pul.period, pul.psi, synth.DT)
        if prod:
            p = B.production(p)
        got = static_search(p, x)
        ref = regular_search(p, x)
        assert_same(got, ref, p)
        # harmonic sums and candidate selection of its own power spectrum are
        # exactly the restated reference's (shaders/harmonic.comp, select)
        assert np.array_equal(got[1], oracle.select(oracle.harmonic(got[0], p), p))
        found += len(ref[1])
    assert found > 0


def test_static_search_rejects_oversized_series():
    n = 1 << 21
    p = B.parameters(n, n - 17, 0.3, 3600.0, 1.1, synth.DT)
    q = as_params(p)
    one = ctypes.c_uint32()
    st = lib().brp_cuda_search_static(ctypes.byref(q), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                      ctypes.c_void_p(16), 1, ctypes.byref(one), ctypes.byref(one), None)
    assert st == 4
    assert b"static scratch bound" in lib().brp_cuda_search_static_error()
