"""Autotuner of the bank search (Python face of brp_cuda_bank_autotune).

For every length class of a bank the C autotuner times, on the device, each
compatible pair of compiled pass-1 / pass-2 configurations (column length,
columns per CTA, threads; row length, row pairs per CTA, threads) with each
number of templates per launch and each number of launch chains, replaying the
captured graph of the bank's own templates with L2 flushed between replays,
and keeps the fastest.  Results are cached in a JSON plan file keyed by
device, length and template count, which the library itself reads for its
default plans (brp_cuda_load_plan_cache).
"""
import ctypes
import json
import os

import numpy as np

from ._lib import BrpError, Params, as_params, fast_configs, lib, ptr

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "brp_b200", "plans.json")
USE_CACHE = 1


class TuneResult(ctypes.Structure):
    """brp_tune_result of include/brp_cuda.h."""
    _fields_ = [("ms", ctypes.c_double), ("n", ctypes.c_uint32), ("pass1", ctypes.c_int32),
                ("pass2", ctypes.c_int32), ("group", ctypes.c_uint32), ("chains", ctypes.c_uint32),
                ("tried", ctypes.c_uint32), ("cached", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


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


def load_cache(path=DEFAULT_CACHE):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def autotune(bank, templates, series_of=None, reps=3, groups=(16, 32, 64, 128), cache_path=DEFAULT_CACHE,
             use_cache=True):
    """Chooses the fastest configuration for every length class of `bank` on
    this workload (brp_cuda_bank_autotune); leaves the bank configured with it
    and returns {n: {"pass1": id, "pass2": id, "group": g, "chains": c,
    "ms": t, "tried": count, "cached": bool}}.  With use_cache the plan file
    is read (an entry for this device, length and template count is reused)
    and updated; without it the file is neither read nor written."""
    arr = templates if isinstance(templates, ctypes.Array) else (Params * len(templates))(
        *[as_params(t) for t in templates])
    count = len(arr)
    so = np.zeros(count, np.uint32) if series_of is None else np.ascontiguousarray(series_of, np.uint32)
    g = np.ascontiguousarray(groups, np.uint32)
    out = (TuneResult * 8)()
    found = ctypes.c_uint32()
    path = cache_path.encode() if use_cache and cache_path else None
    L = lib()
    st = L.brp_cuda_bank_autotune(bank._b, arr, ptr(so), count, reps, ptr(g), g.size, path,
                                  USE_CACHE if use_cache else 0, out, len(out), ctypes.byref(found))
    if st:
        raise BrpError(st, L.brp_cuda_autotune_error().decode())
    return {int(r.n): {"pass1": r.pass1, "pass2": r.pass2, "group": r.group, "chains": r.chains, "ms": r.ms,
                       "tried": r.tried, "cached": bool(r.cached)} for r in out[:found.value]}


def _device_key():
    """The plan file's device key of the current CUDA device."""
    import torch
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return "%s/sm%d%d/%d" % (p.name, p.major, p.minor, p.multi_processor_count)


def load_plans(path=None):
    """Makes the library's default plans follow a plan file (None: the default
    file; "": forget all plans and use the built-in pairs)."""
    L = lib()
    st = L.brp_cuda_load_plan_cache(None if path is None else path.encode())
    if st:
        raise BrpError(st, L.brp_cuda_autotune_error().decode())
