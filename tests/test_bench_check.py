"""bench.py's parity check against the reference's CPU path, on the CPU: the
bench's own workload (N = 2^22), two templates, with a stand-in for the bank
that returns the reference's lists (every count must then agree) and one that
drops a candidate far from a threshold and perturbs a power (the check must
report both)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402
import brp_b200 as B  # noqa: E402


class ListBank:
    """Returns fixed candidate lists from run_flat, like Bank.run_flat."""

    def __init__(self, lists):
        self.lists = lists
        self.rows = None

    def set_toplist_filter(self, rows):
        self.rows = rows

    def run_flat(self, arr):
        n = len(arr)
        lists = [np.asarray(c).view(B.CANDIDATE) for c in self.lists[:n]]
        counts = np.array([len(c) for c in lists], np.uint32)
        offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
        return np.concatenate(lists), offs, counts, np.zeros(n, np.uint32)


@pytest.fixture(scope="module")
def setup(oracle):
    wl = bench.workload(2)
    pool = bench.cpu_pool(wl.series[0], 2)
    ref = pool.map(bench._cpu_check, [bytes(wl.templates[k]) for k in range(2)])
    yield wl, pool, ref
    pool.close()


def test_check_agrees_with_itself(setup):
    wl, pool, ref = setup
    bank = ListBank([r[1] for r in ref])
    out = bench.reference_check(B, bank, pool, wl.templates, np.asarray(wl.orbits, np.float64), 2, ref[0][0])
    assert bank.rows == 0  # the bank's lists are taken with the pre-filter off
    assert out["resampled_template0_bit_exact"] and out["status_words_clear"]
    assert out["candidates_gpu"] == out["candidates_reference"] > 0
    assert out["candidates_differ"] == 0 and out["max_power_rel_diff_shared"] == 0.0
    assert out["toplist_row_order_equal"] and out["toplist_rows"] > 0


def test_check_reports_differences(setup):
    wl, pool, ref = setup
    lists = [np.array(r[1]).view(B.CANDIDATE).copy() for r in ref]
    thr = wl.templates[0].threshold
    c = lists[0]
    far = int(np.argmax(c["power"] / np.array([thr[int(l)] for l in c["level"]])))
    lists[0] = np.delete(c, far)
    lists[1]["power"][0] *= np.float32(1.001)
    out = bench.reference_check(B, ListBank(lists), pool, wl.templates, np.asarray(wl.orbits, np.float64), 2,
                                "0" * 40)
    assert not out["resampled_template0_bit_exact"]
    assert out["candidates_differ"] == 1 and out["candidates_differ_away_from_threshold"] == 1
    assert out["max_power_rel_diff_shared"] > 9e-4


def test_reference_arm_templates_equal_the_cuda_arms(oracle):
    """The reference arm builds its bank with the reference's own
    search_parameters; the templates are byte-identical to the CUDA arm's
    (this package's host code), so both arms search the same bank."""
    from brp_b200 import synth
    mine = synth.bank_workload("t", [1 << 16], [24], [1], seed=3)
    ref = synth.bank_workload("t", [1 << 16], [24], [1], seed=3, search=bench.reference_search())
    assert [bytes(p) for p in mine.templates] == [bytes(p) for p in ref.templates]
    assert np.array_equal(mine.series[0], ref.series[0])


def test_reference_arm_runs_without_the_cuda_library(tmp_path):
    """`bench.py --impl reference` (a small bank) prints its line and never maps
    this repository's CUDA library into the process."""
    import json
    import subprocess
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--templates', '8', '--steps', '1', "
            "'--warmup', '1']; runpy.run_path(%r, run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); print('MAPPED' if 'libbrp_cuda' in maps else 'CLEAN')"
            % os.path.join(ROOT, "bench.py"))
    out = subprocess.run([sys.executable, "-c", code], cwd=str(tmp_path), capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "CLEAN"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["config"]["templates_per_step"] == 8
    assert line["config"]["workload"] == bench.workload_name(8)
    assert line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
