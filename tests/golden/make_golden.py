"""Generates the golden vectors of tests/golden/ from the reference's own CPU
code (src/science.cpp and src/workload.cpp compiled into oracle/_ref by
`make -C oracle ref`).  Run here, where the reference sources exist:

    python tests/golden/make_golden.py

The vectors pin the oracle (oracle/brp_oracle.c) and the product's host code
to the reference: LUT sine, template constants, resampling indices, search
parameters, harmonic sums, the full per-template pipeline and the toplist.
Inputs are seeded synthetic data; the FFT inside the reference pipeline is the
FP64 DFT stand-in for FFTW (oracle/ref_shims/ref_shims.cpp).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT]
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "reference_vectors.npz")
DT = 128e-6


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libbrp_ref.so missing: run `make -C oracle ref` first")
    R = O.ref()
    rng = np.random.default_rng(2024)
    out = {}

    # LUT sine (src/science.cpp:20-28) over a wide phase range
    xs = np.concatenate([rng.uniform(-2e4, 2e4, 3000), rng.uniform(-10, 10, 1000),
                         np.arange(-64, 65) * (6.283185 / 64)]).astype(np.float32)
    out["lut_x"] = xs
    out["lut_sin"] = np.array([R.ref_lut_sin(float(x)) for x in xs], np.float32)

    # template constants (src/science.cpp:46-65) + production variant, and resampling indices
    cases = [(64, 47, 0.0, 10.0, 0.0, 1e-3), (96, 64, 1e-3, 1.0, 6.2, 1e-3), (4096, 4079, 0.002, 120.0, 0.3, 0.000256),
             (8192, 8000, 0.9, 600.0, -1.7, DT), (3 * 4096, 3 * 4096 - 5, 2.5, 3600.0, 4.4, DT),
             (65536, 65519, 0.3, 3600.0, 1.1, DT), (65536, 65519, 3.0, 3600.0, 5.9, DT)]
    params, prod, idx, idx_prod = [], [], [], []
    for c in cases:
        p = O.ref_parameters(*c)
        params.append(np.frombuffer(bytes(p), np.uint8))
        x = np.arange(p.unpadded, dtype=np.float32)
        idx.append(O.ref_resample(x, p)[:p.steps].astype(np.int32))
        q = O.Params.from_buffer_copy(bytes(p))
        q.flags = 6
        q.s0 = np.float32(np.float32(q.tau) * np.sin(np.float32(q.psi))) * np.float32(q.step_inv)
        q = O.ref_resampling_steps(q)
        prod.append(np.frombuffer(bytes(q), np.uint8))
        idx_prod.append(O.ref_resample(x, q)[:q.steps].astype(np.int32))
    out["param_cases"] = np.array(cases, np.float64)
    out["params"] = np.stack(params)
    out["params_production"] = np.stack(prod)
    for k in range(len(cases)):
        out["index_%d" % k] = idx[k]
        out["index_production_%d" % k] = idx_prod[k]

    # search parameters (src/workload.cpp:108-125)
    sp_cases = [(1 << 22, 1 << 22, 128.0, 3600.0 * 5, 1.2, 0.7, 400.0, 0.08, 1000),
                (3 << 20, 3 << 20, 128.0, 86000.0, 2.9, 4.0, 800.0, 0.01, 500),
                (1 << 20, 900000, 64.0, 20000.0, 0.0, 0.0, 50.0, 1e-6, 7),
                (1 << 17, 1 << 17, 128.0, 4000.0, 0.9, 1.3, 400.0, 0.08, 1000)]
    out["search_cases"] = np.array(sp_cases, np.float64)
    out["search_params"] = np.stack([np.frombuffer(bytes(O.ref_search_parameters(*c)), np.uint8) for c in sp_cases])

    # harmonic sums on random power spectra with assorted ranges
    hs = []
    for k, (M, window, fund, harm) in enumerate([(4096, 8, 4096, 4096), (4096, 100, 700, 3000),
                                                 (6144, 3, 6144, 5000), (2048, 50, 60, 2048)]):
        P = rng.exponential(1.0, M).astype(np.float32)
        P[rng.integers(0, M, 20)] *= 40
        P[0] = 0
        p = O.ref_parameters(2 * M, 2 * M - 17, 0.1, 3600.0, 0.1, DT)
        p.window, p.fundamental, p.harmonic = window, fund, harm
        for h, t in enumerate([6.0, 9.0, 14.0, 22.0, 38.0]):
            p.threshold[h] = t
        out["hs_power_%d" % k] = P
        out["hs_params_%d" % k] = np.frombuffer(bytes(p), np.uint8)
        out["hs_summed_%d" % k] = O.ref_harmonic(P, p)
        hs.append(k)

    # full reference pipeline (src/science.cpp:113-120) on a small synthetic case
    n = 8192
    t = np.arange(n - 17) * DT
    x = (rng.standard_normal(n - 17) + 0.4 * np.cos(2 * np.pi * 211.0 * (t + 0.01 * np.sin(2 * np.pi * t / 600.0)))
         ).astype(np.float32)
    p = O.ref_parameters(n, n - 17, 0.01, 600.0, 0.0, DT)
    r = O.ref_reference(x, p)
    out["pipe_input"] = x
    out["pipe_params"] = np.frombuffer(bytes(p), np.uint8)
    for key in ("resampled", "power", "summed", "candidates"):
        out["pipe_" + key] = r[key]

    # toplist (src/workload.cpp:126-159) after a seeded candidate sequence
    p = O.ref_search_parameters(1 << 20, 1 << 20, 128.0, 3600.0, 0.5, 0.1, 400.0, 0.08, 1000)
    tl = O.RefToplist()
    seq = []
    for tpl in range(120):
        cnt = int(rng.integers(0, 30))
        c = np.zeros(cnt, O.CANDIDATE)
        c["bin"] = rng.integers(p.window, p.fundamental, cnt)
        c["level"] = rng.integers(0, 5, cnt)
        thr = np.asarray(list(p.threshold))
        c["power"] = (thr[c["level"]] * rng.uniform(0.9, 3.0, cnt)).astype(np.float32)
        c = c[np.lexsort((c["bin"], c["level"]))]
        orb = (3600.0 + tpl, 0.01 * tpl, 0.05 * tpl)
        q = tl.thresholds(p)
        tl.retain(c, *orb, q)
        seq.append((c, orb))
    out["top_params"] = np.frombuffer(bytes(p), np.uint8)
    out["top_cands"] = np.concatenate([c for c, _ in seq])
    out["top_counts"] = np.array([len(c) for c, _ in seq], np.int64)
    out["top_orbits"] = np.array([o for _, o in seq], np.float64)
    out["top_final"] = tl.final()
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
