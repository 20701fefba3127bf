"""The multi-rank bank flow on real kernels: two ranks (processes, gloo
process group) on one GPU each search their contiguous template shard with
Bank.run_flat, gather their kept candidate lists to rank 0, and rank 0 folds
the bank-wide toplist (brp_b200.shard.search_and_fold, the step bench.py runs
under torchrun).  The toplist must equal the one-rank run's (batch
invariance, src/workunit_main.cpp:85-93).  The ranks' kernels never wait on
one another (no device-side collective), so sharing one GPU is safe."""
import datetime
import os
import socket
import sys
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "boinc-einstein-bpr4-v3d_b200")


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def workload():
    from brp_b200 import synth
    return synth.bank_workload("multirank", [1 << 20], [24], [2], seed=51, f0=800.0, sigmas=(5.0,))


def search(bank_filter, rank, world):
    """This rank's end-to-end step (toplist on rank 0, None elsewhere)."""
    import brp_b200 as B
    from brp_b200 import shard
    wl = workload()
    begin, end = shard.shard_range(len(wl.templates), rank, world)
    bank = B.Bank(wl.n, [len(x) for x in wl.series], end - begin, 8192, device=0)
    bank.set_series(0, wl.series[0])
    if bank_filter:
        bank.set_toplist_filter(100)
    top = shard.search_and_fold(bank, B.Bank.params_array(wl.templates[begin:end]), begin,
                                B.Bank.params_array(wl.templates), np.asarray(wl.orbits, np.float64))
    bank.close()
    return None if top is None else top.final()


def _worker(rank, world, port, outdir, bank_filter):
    sys.path[:0] = [ROOT, PKG]
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        top = search(bank_filter, rank, world)
        if rank == 0:
            np.save(os.path.join(outdir, "top.npy"), top)
        open(os.path.join(outdir, "ok-%d" % rank), "w").close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bank_filter", [False, True])
def test_two_ranks_on_one_gpu_equal_one_rank(bank_filter):
    import torch.multiprocessing as mp
    outdir = tempfile.mkdtemp()
    mp.spawn(_worker, args=(2, free_port(), outdir, bank_filter), nprocs=2, join=True)
    assert os.path.exists(os.path.join(outdir, "ok-0")) and os.path.exists(os.path.join(outdir, "ok-1"))
    two = np.load(os.path.join(outdir, "top.npy"))
    one = search(bank_filter, 0, 1)
    assert len(one) > 0
    assert two.tobytes() == one.tobytes()


def test_bench_multirank_path_on_one_gpu():
    """bench.py's own multi-rank path under torchrun (two gloo ranks sharing
    the GPU): template shards, barriers, max-over-ranks timing and the
    end-to-end step with the gather to rank 0 and the bank-wide fold."""
    import json
    import subprocess
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.join(ROOT, "bench.py"),
           "--gpus", "2", "--dist-backend", "gloo", "--same-device", "--templates", "16", "--steps", "2",
           "--warmup", "3", "--no-cpu-baseline", "--no-plain", "--no-tune"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = lines[0]
    assert line["n_gpus"] == 2 and line["config"]["parallelism"] == "template shards, 2 rank(s)"
    assert line["config"]["templates_per_gpu"] == 16 and line["value"] > 0 and line["e2e"]["value"] > 0
