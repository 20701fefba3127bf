"""The autotuner for C callers (brp_cuda_bank_autotune) and its plan file.

* The C autotuner times the compiled pass pairs, group sizes and chain counts of
  a bank at n = 2^21 -- a length without a built-in preferred pair -- leaves the
  bank configured with the fastest, and records it in a JSON plan file keyed by
  device, length and template count.
* The Python tuner (brp_b200.tune, the same autotuner) reuses that entry from
  the file without timing.
* After the library loads the file, brp::GPU (brp_cuda_create, the reference's
  brp_bench / brp_workunit path) takes the tuned pass pair for that length, and
  its candidates equal the tuned bank's.
* A plan file written by Python's json module with a chosen pair steers the
  library's default choice the same way (the format is shared both ways).
"""
import json

import numpy as np
import pytest

import brp_b200 as B
from brp_b200 import synth, tune

pytestmark = pytest.mark.gpu
N = 1 << 21


@pytest.fixture(scope="module")
def workload():
    return synth.bank_workload("tune-2^21", [N], [32], [1], seed=61, f0=800.0, sigmas=(5.0,))


def gpu_passes(p, x):
    g = B.GPU(p, x, 256, 0, 1, stockham=True, packed=True)
    info = g.device_info()
    g.set_template(p)
    g.run()
    cands = g.candidates()
    g.close()
    fields = dict(kv.split("=") for kv in info.split("; ") if "=" in kv)
    return int(fields["pass1"]), int(fields["pass2"]), cands


def test_c_autotuner_plan_file_and_default_plans(tmp_path, workload):
    wl = workload
    path = str(tmp_path / "plans.json")
    bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    bank.set_series(0, wl.series[0])
    res = tune.autotune(bank, wl.templates, reps=2, groups=(16, 32), cache_path=path)
    r = res[N]
    assert not r["cached"] and r["tried"] >= 8 and r["group"] in (16, 32) and r["chains"] in (1, 2)
    tuned, _, status = bank.run(wl.templates)
    assert not status.any()
    plans = json.load(open(path))
    keys = [k for k in plans if k.endswith("|n=%d|templates=%d" % (N, len(wl.templates)))]
    assert len(keys) == 1
    entry = plans[keys[0]]
    assert (entry["pass1"], entry["pass2"], entry["group"], entry["chains"]) == \
           (r["pass1"], r["pass2"], r["group"], r["chains"])
    # the same file through the Python face: reused without timing
    again = tune.autotune(bank, wl.templates, reps=2, groups=(16, 32), cache_path=path)[N]
    assert again["cached"] and (again["pass1"], again["pass2"]) == (r["pass1"], r["pass2"])
    bank.close()
    # brp::GPU's default plan for n = 2^21 is the tuned pair, with the same candidates
    tune.load_plans(path)
    p1, p2, cands = gpu_passes(wl.templates[0], wl.series[0])
    assert (p1, p2) == (r["pass1"], r["pass2"])
    assert np.array_equal(cands, tuned[0])


def near_threshold_only(a, b, p, rtol=1e-5):
    ka = {(int(x), int(y)) for x, y in zip(a["bin"], a["level"])}
    kb = {(int(x), int(y)) for x, y in zip(b["bin"], b["level"])}
    va = {(int(x), int(y)): float(v) for x, y, v in zip(a["bin"], a["level"], a["power"])}
    vb = {(int(x), int(y)): float(v) for x, y, v in zip(b["bin"], b["level"], b["power"])}
    return all(abs(va.get(k, vb.get(k)) - float(p.threshold[k[1]])) <= rtol * float(p.threshold[k[1]])
               for k in ka ^ kb)


def test_python_written_plan_file_steers_the_default_choice(tmp_path, workload):
    wl = workload
    p, x = wl.templates[0], wl.series[0]
    key = "%s|n=%d|templates=%d" % (tune._device_key(), N, 100000)  # the largest bank's entry wins
    try:
        tune.load_plans("")  # built-in choice first
        _, _, ref = gpu_passes(p, x)
        for pair in ((117, 201), (110, 203)):
            path = str(tmp_path / ("plans-%d.json" % pair[0]))
            with open(path, "w") as f:
                json.dump({key: {"pass1": pair[0], "pass2": pair[1], "group": 16, "chains": 1, "ms": 1.0}}, f,
                          indent=1, sort_keys=True)
            tune.load_plans(path)
            p1, p2, cands = gpu_passes(p, x)
            assert (p1, p2) == pair
            assert len(cands) > 0 and near_threshold_only(cands, ref, p)
    finally:
        tune.load_plans("")  # later tests get the built-in pairs


def test_bank_created_under_a_two_chain_plan(tmp_path, workload):
    """A new bank takes the cached plan's templates per launch and chains
    (each chain with its own intermediate buffers) and finds exactly what a
    bank configured with the same plan by hand finds."""
    wl = workload
    key = "%s|n=%d|templates=%d" % (tune._device_key(), N, 100000)
    path = str(tmp_path / "plans-chains.json")
    with open(path, "w") as f:
        json.dump({key: {"pass1": 117, "pass2": 201, "group": 8, "chains": 2, "ms": 1.0}}, f)
    try:
        tune.load_plans(path)
        bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
        bank.set_series(0, wl.series[0])
        got, _, status = bank.run(wl.templates)
        assert not status.any() and bank.kernels_per_run == 3 * 4 + 1  # 32 templates in 4 groups of 8
        bank.close()
    finally:
        tune.load_plans("")
    ref_bank = B.Bank(wl.n, [len(x) for x in wl.series], len(wl.templates), 8192)
    ref_bank.set_series(0, wl.series[0])
    ref_bank.configure(N, pass1=117, pass2=201, group=8, chains=2)
    ref, _, _ = ref_bank.run(wl.templates)
    ref_bank.close()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
