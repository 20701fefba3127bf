"""The reference's own drivers, unmodified, on the CUDA backend.

oracle/_ref/brp_bench is src/main.cpp and oracle/_ref/brp_workunit is
src/workunit_main.cpp of the reference, linked with the brp::GPU adapter
(csrc/brp_gpu_adapter.cpp) over libbrp_cuda.so (oracle/Makefile, target
dropin).  They apply the reference's own validation gates (src/main.cpp:55-94,
src/workunit_main.cpp:103-122) and exit 0 only when every gate passes.  The
binaries are built where the reference sources are present; elsewhere these
tests are skipped."""
import gzip
import json
import os
import subprocess

import numpy as np
import pytest

import dd_files
from brp_b200 import synth

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "oracle", "_ref", "brp_bench")
WORKUNIT = os.path.join(ROOT, "oracle", "_ref", "brp_workunit")


def need(path):
    if not os.path.exists(path):
        pytest.skip("drop-in binary absent (built from the reference sources by `make -C oracle dropin`)")


@pytest.mark.parametrize("flags", [
    [],
    ["--stockham", "--tile", "0", "--packed", "--batch", "4"],
    ["--stockham", "--tile", "0", "--radix8-store", "--packed", "--fused-power", "--scatter", "--production"],
    ["--n", "196608", "--stockham", "--tile", "0", "--radix4", "--packed"],
    ["--n", "1048576", "--stockham", "--tile", "0", "--packed", "--production", "--tau", "0.8", "--period", "3000"],
])
def test_brp_bench_valid(flags):
    need(BENCH)
    r = subprocess.run([BENCH, "--reps", "3"] + flags, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout)
    assert out["valid"] and out["index_mismatches"] == 0 and out["candidate_mismatches"] == 0
    assert out["harmonic_isolated_l2"] == 0.0


def _workunit_inputs(tmp_path, n=1 << 17, templates=24):
    rng = np.random.default_rng(17)
    pul = synth.Pulsar(223.0, 4000.0, 0.9, 1.3, 0.03, 8, 0.1)
    x = synth.make_series(n, 9, [pul])
    dd = tmp_path / "obs.binary"
    dd_files.write_dd(dd, np.clip(np.round(x * 8), -127, 127).astype(np.int8), 128.0, 8.0)
    pre = tmp_path / "pre.f32"
    dd_files.write_floats(pre, x)
    orbits = synth.random_orbits(rng, templates, 1.0, 3.0, 1.5)
    orbits[5] = (pul.period, pul.tau, pul.psi)
    bank = tmp_path / "bank.txt"
    dd_files.write_bank(bank, orbits)
    return dd, pre, bank


def _run_workunit(tmp_path, dd, pre, bank, tag, extra):
    out, met = tmp_path / ("cand-%s.txt" % tag), tmp_path / ("met-%s.jsonl" % tag)
    cmd = [WORKUNIT, "--input", str(dd), "--bank", str(bank), "--zap", "unused", "--padding", "1",
           "--f0", "400", "--false-alarm", "0.08", "--window", "1000", "--output", str(out), "--metrics", str(met),
           "--preprocessed", str(pre)] + extra
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), out.read_text()


def test_brp_workunit_validated_and_toplist_equals_cpu(tmp_path):
    need(WORKUNIT)
    dd, pre, bank = _workunit_inputs(tmp_path)
    v, _ = _run_workunit(tmp_path, dd, pre, bank, "validate", ["--validate", "--batch", "1", "--packed"])
    assert v["valid"]
    g, gpu_top = _run_workunit(tmp_path, dd, pre, bank, "gpu", ["--batch", "8", "--packed", "--radix8",
                                                                 "--fused-power", "--scatter"])
    c, cpu_top = _run_workunit(tmp_path, dd, pre, bank, "cpu", ["--cpu"])
    assert g["candidates"] == c["candidates"] > 0
    rows_g, rows_c = _rows(gpu_top), _rows(cpu_top)
    assert len(rows_g) == len(rows_c)
    for a, b in zip(rows_g, rows_c):
        assert a[:4] == b[:4] and a[6] == b[6]          # frequency, orbit, harmonics
        assert abs(a[4] - b[4]) <= 1e-4 * abs(b[4])     # power (6 significant digits printed)
        assert abs(a[5] - b[5]) <= 1e-4 * abs(b[5]) + 1e-3


def _rows(text):
    out = []
    for line in text.splitlines():
        if line.startswith("%"):
            continue
        f = line.split()
        out.append((f[0], f[1], f[2], f[3], float(f[4]), float(f[5]), f[6]))
    return out


def test_brp_workunit_accepts_gpu_whitening(tmp_path):
    """The reference's own workunit driver whitens on the CPU (src/workunit_main.cpp:54,
    brp::preprocess with the oracle's FFT/median/RNG stand-ins) and checks a
    reference folder with its own gate (:57-62: decoded bit-exact, preprocessed
    relative L2 < 1e-4); the folder holds the GPU's decoding and whitening."""
    need(WORKUNIT)
    from brp_b200 import whiten
    dd, _, bank = _workunit_inputs(tmp_path)
    zap = tmp_path / "zap.txt"
    zap.write_text("223.0 223.05\n446.0 446.1\n1200 1200\n")
    raw = np.frombuffer(gzip.open(dd).read()[1168:], np.uint8)
    n = len(raw)
    dec, pre = whiten.preprocess_dd(raw, n, False, 8.0, n, 128.0, 1.0, 1000, str(zap))
    ref = tmp_path / "ref"
    ref.mkdir()
    dd_files.write_floats(ref / "decoded.f32", dec)
    dd_files.write_floats(ref / "preprocessed.f32", pre)
    out, met = tmp_path / "cand-white.txt", tmp_path / "met-white.jsonl"
    cmd = [WORKUNIT, "--input", str(dd), "--bank", str(bank), "--zap", str(zap), "--padding", "1", "--f0", "400",
           "--false-alarm", "0.08", "--window", "1000", "--output", str(out), "--metrics", str(met),
           "--reference-dir", str(ref), "--cpu"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    m = json.loads(r.stdout.strip().splitlines()[-1])
    print("workunit gate: decoded_l2 %g, preprocessed_l2 %g" % (m["decoded_l2"], m["preprocessed_l2"]))
    assert m["decoded_l2"] == 0 and m["preprocessed_l2"] < 2e-6
