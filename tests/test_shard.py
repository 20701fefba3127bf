"""Multi-rank bank search on CPU (gloo, world size 2): template shards, the
candidate gather to rank 0 and the bank-wide toplist, which must equal the
single-process toplist (batch invariance).  Each rank computes its shard's
candidates with the CPU oracle here; on GPUs the same host logic wraps
Bank.run.  A second test makes one rank fail before the gather and checks
that the other rank's collective ends with an error instead of waiting."""
import datetime
import os
import socket
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "boinc-einstein-bpr4-v3d_b200")


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def small_bank():
    from brp_b200 import synth
    return synth.bank_workload("shard-test", [1 << 16], [11], [1], seed=31, f0=800.0, sigmas=(3.5,))


def _worker(rank, world, port, outdir, fail_rank):
    sys.path[:0] = [ROOT, PKG]
    import torch.distributed as dist
    from brp_b200 import shard
    from oracle import oracle as O
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=8))
    wl = small_bank()
    begin, end = shard.shard_range(len(wl.templates), rank, world)
    mine = [O.pipeline(wl.series[0], p)["candidates"] for p in wl.templates[begin:end]]
    try:
        if rank == fail_rank:
            raise RuntimeError("injected failure before the gather")
        merged = shard.gather_candidates(mine, begin)
        if rank == 0:
            import brp_b200 as B
            top = shard.fold_toplist(B.Toplist(), wl.templates, wl.orbits, merged).final()
            np.save(os.path.join(outdir, "top.npy"), top)
        open(os.path.join(outdir, "ok-%d" % rank), "w").close()
    except Exception as e:  # recorded for the parent test
        open(os.path.join(outdir, "err-%d" % rank), "w").write(str(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _spawn(fail_rank):
    import torch.multiprocessing as mp
    outdir = tempfile.mkdtemp()
    mp.spawn(_worker, args=(2, free_port(), outdir, fail_rank), nprocs=2, join=True)
    return outdir


def test_shard_ranges_cover_bank():
    from brp_b200 import shard
    for count in (1, 7, 512, 1000):
        for world in (1, 2, 3, 8):
            r = [shard.shard_range(count, k, world) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            assert max(e - b for b, e in r) - min(e - b for b, e in r) <= 1


def test_two_rank_toplist_equals_single_process(oracle):
    outdir = _spawn(fail_rank=-1)
    assert os.path.exists(os.path.join(outdir, "ok-0")) and os.path.exists(os.path.join(outdir, "ok-1"))
    top = np.load(os.path.join(outdir, "top.npy"))
    from brp_b200 import shard
    import brp_b200 as B
    wl = small_bank()
    cands = [oracle.pipeline(wl.series[0], p)["candidates"] for p in wl.templates]
    ref = shard.fold_toplist(B.Toplist(), wl.templates, wl.orbits, cands).final()
    assert len(ref) > 0 and top.tobytes() == ref.tobytes()


def test_failed_rank_is_detected():
    outdir = _spawn(fail_rank=1)
    assert os.path.exists(os.path.join(outdir, "err-1"))
    # rank 0's gather ends with an error (peer gone / timeout) instead of hanging
    assert os.path.exists(os.path.join(outdir, "err-0"))
