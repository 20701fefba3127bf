"""Generates tests/golden/whitening_vectors.npz from the reference's own CPU
code (src/workload.cpp compiled into oracle/_ref by `make -C oracle ref`, with
the oracle's stand-ins for FFTW, rngmed and GSL).  Run here, where the
reference sources exist:

    python tests/golden/make_whitening_golden.py

The vectors pin the whitening and RFI zapping of brp::preprocess
(src/workload.cpp:58-95) and the DD sample decoding of brp::load_observation
(:29-57) without the reference library: two preprocess cases (a power-of-two
and a 3*2^k length, overlapping zap ranges in the first) and one int8 and one
packed 4-bit DD file.  Inputs are seeded synthetic data.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.dirname(HERE)]
from oracle import oracle as O  # noqa: E402
from dd_files import write_dd_bytes  # noqa: E402

OUT = os.path.join(HERE, "whitening_vectors.npz")
SAMPLE_US = 128.0
# (n, samples, window, zap rows (lower, upper) in the reference's units)
PREPROCESS_CASES = [
    (1 << 15, 30000, 1000, [(50.0, 50.6), (50.4, 51.0), (711.0, 711.2)]),
    (3 << 13, 20000, 64, [(1200.0, 1201.5)]),
]


def series(samples, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(samples).astype(np.float32)
    t = np.arange(samples) * SAMPLE_US * 1e-6
    x += (0.3 * np.sin(2 * np.pi * 50.7 * t) + 0.2 * np.sin(2 * np.pi * 711.1 * t)).astype(np.float32)
    return x


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libbrp_ref.so missing: run `make -C oracle ref` first")
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for k, (n, samples, window, rows) in enumerate(PREPROCESS_CASES):
            x = series(samples, 100 + k)
            zap = os.path.join(tmp, "zap%d.txt" % k)
            with open(zap, "w") as f:
                f.write("".join("%r %r\n" % r for r in rows))
            out["pre_input_%d" % k] = x
            out["pre_case_%d" % k] = np.array([n, samples, window, n / samples], np.float64)
            out["pre_zap_%d" % k] = np.array(rows, np.float64).reshape(-1, 2)
            out["pre_output_%d" % k] = O.ref_preprocess(x, n, SAMPLE_US, n / samples, zap, window)
        rng = np.random.default_rng(77)
        for name, packed, samples in (("int8", False, 2048), ("packed", True, 2048)):
            raw = rng.integers(0, 256, samples // 2 if packed else samples, dtype=np.uint8)
            path = os.path.join(tmp, "obs." + ("bin4" if packed else "binary"))
            write_dd_bytes(path, raw, samples, SAMPLE_US, scale=3.5)
            meta, decoded = O.ref_load_observation(path, 1.0)
            out["dd_raw_" + name] = raw
            out["dd_meta_" + name] = np.array(meta, np.float64)
            out["dd_decoded_" + name] = decoded
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
