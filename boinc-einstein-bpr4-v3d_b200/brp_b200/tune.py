"""Autotuner of the bank search.

For every length class of a bank it times, on the device, each compatible
pair of compiled pass-1 / pass-2 configurations (column length, columns per
CTA, threads; row length, row pairs per CTA, threads) and each number of
templates per launch, replaying the captured graph of the bank's own
templates with L2 flushed between replays, and keeps the fastest.  Results
are cached in a JSON plan file keyed by device, length and template count.
"""
import json
import os

import numpy as np

from ._lib import fast_configs

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "brp_b200", "plans.json")


def candidates(n, groups=(4, 8, 16), chains=(1, 2)):
    """(pass1 id, pass2 id, group, chains) whose decomposition covers length n."""
    M = n // 2
    cfg = fast_configs()
    p1 = [(i, L) for i, L, k in cfg if k == 1]
    p2 = [(i, L) for i, L, k in cfg if k == 2]
    out = []
    for i1, L1 in p1:
        for i2, L2 in p2:
            if L1 * L2 == M:
                for g in groups:
                    for c in chains:
                        out.append((i1, i2, g, c))
    return out


def _device_key():
    try:
        import torch
        p = torch.cuda.get_device_properties(torch.cuda.current_device())
        return "%s/sm%d%d/%d" % (p.name, p.major, p.minor, p.multi_processor_count)
    except Exception:
        return "cuda"


def load_cache(path=DEFAULT_CACHE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(cache, path=DEFAULT_CACHE):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def time_replays(bank, reps, flush):
    """Mean device time (ms) of `reps` graph replays, L2 flushed before each."""
    import torch
    stream = torch.cuda.ExternalStream(bank.stream)
    total = 0.0
    for _ in range(reps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bank.launch()
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total / reps


def autotune(bank, templates, series_of=None, reps=3, groups=(16, 32, 64, 128), chains=(1, 2), cache_path=DEFAULT_CACHE,
             use_cache=True):
    """Chooses the fastest configuration for every length class of `bank` on
    this workload; leaves the bank configured with it and returns
    {n: {"pass1": id, "pass2": id, "group": g, "ms": t, "tried": [...]}}."""
    import torch
    so = np.zeros(len(templates), np.uint32) if series_of is None else np.asarray(series_of, np.uint32)
    lengths = sorted({int(bank.n[s]) for s in so})
    cache = load_cache(cache_path) if use_cache else {}
    dev = _device_key()
    flush = torch.empty((512 << 20) // 4, dtype=torch.float32, device="cuda")
    result = {}
    for n in lengths:
        key = "%s|n=%d|templates=%d" % (dev, n, len(templates))
        if use_cache and key in cache:
            c = cache[key]
            bank.configure(n, c["pass1"], c["pass2"], c["group"], c.get("chains", 1))
            result[n] = dict(c, cached=True)
            continue
        tried = []
        for i1, i2, g, ch in candidates(n, groups, chains):
            try:
                bank.configure(n, i1, i2, g, ch)
                bank.run(templates, so)
                ms = time_replays(bank, reps, flush)
            except Exception as e:  # a configuration that does not fit this device
                tried.append({"pass1": i1, "pass2": i2, "group": g, "chains": ch, "error": str(e)})
                continue
            tried.append({"pass1": i1, "pass2": i2, "group": g, "chains": ch, "ms": ms})
        ok = [t for t in tried if "ms" in t]
        if not ok:
            bank.configure(n, 0, 0, 0, 0)
            continue
        best = min(ok, key=lambda t: t["ms"])
        bank.configure(n, best["pass1"], best["pass2"], best["group"], best["chains"])
        result[n] = dict(best, tried=tried)
        cache[key] = {k: best[k] for k in ("pass1", "pass2", "group", "chains", "ms")}
    if use_cache:
        save_cache(cache, cache_path)
    del flush
    return result
