"""Host-side functions of the search path, through the C ABI: template
constants (src/science.cpp:41-65), production search parameters
(src/workload.cpp:108-125) and the bank-wide toplist (src/workload.cpp:126-159)."""
import ctypes

import numpy as np

from ._lib import BANK_CANDIDATE, CANDIDATE, BrpError, Params, as_params, lib, ptr


def _err():
    return lib().brp_cuda_last_error(None).decode()


def parameters(n, unpadded, tau, period, psi, dt):
    """brp::parameters: bench-mode template constants (window 8, thresholds 20/30/45/70/110)."""
    p = Params()
    st = lib().brp_host_parameters(n, unpadded, float(np.float32(tau)), float(np.float32(period)),
                                   float(np.float32(psi)), float(np.float32(dt)), ctypes.byref(p))
    if st:
        raise BrpError(st, "invalid observation/template")
    return p


def resampling_steps(p):
    q = as_params(p)
    st = lib().brp_host_resampling_steps(ctypes.byref(q))
    if st:
        raise BrpError(st, "template produces empty series")
    return q


def production(p):
    """src/main.cpp:41: FMA resampling arithmetic (flags 2|4) with the float-sine S0."""
    q = as_params(p)
    q.flags = 2 | 4
    q.s0 = np.float32(np.float32(q.tau) * np.sin(np.float32(q.psi))) * np.float32(q.step_inv)
    return resampling_steps(q)


def search_parameters(n, samples, sample_us, period, tau, psi, f0=400.0, false_alarm=0.08, window=1000):
    """brp::search_parameters for an observation of `samples` samples padded to n."""
    p = Params()
    st = lib().brp_host_search_parameters(n, samples, sample_us, period, tau, psi, f0, false_alarm, window,
                                          ctypes.byref(p))
    if st:
        raise BrpError(st, "invalid search parameters")
    return p


class Toplist:
    """brp::Toplist: 5 harmonic levels x 100 rows, final ranking by significance."""

    def __init__(self):
        self._t = lib().brp_toplist_create()
        if not self._t:
            raise MemoryError("toplist allocation failed")

    def __del__(self):
        if getattr(self, "_t", None):
            lib().brp_toplist_destroy(self._t)
            self._t = None

    def thresholds(self, p):
        q = as_params(p)
        lib().brp_toplist_thresholds(self._t, ctypes.byref(q))
        return q

    def retain(self, candidates, period, tau, psi, p):
        c = np.ascontiguousarray(candidates, dtype=CANDIDATE)
        st = lib().brp_toplist_retain(self._t, ptr(c), c.size, period, tau, psi, ctypes.byref(as_params(p)))
        if st:
            raise BrpError(st, "invalid compact candidate")

    def fold(self, templates, orbits, candidates, counts=None):
        """Thresholds + retain for every template in bank order, in one call.
        `candidates` is a list of per-template arrays, or (with `counts`) the
        flat array of Bank.run_flat; `templates` a list or a Params array."""
        arr = templates if isinstance(templates, ctypes.Array) else \
            (Params * len(templates))(*[as_params(t) for t in templates])
        count = len(arr)
        orb = np.ascontiguousarray(orbits, dtype=np.float64).reshape(count, 3)
        if counts is None:
            counts = np.array([len(c) for c in candidates], np.uint32)
            flat = np.ascontiguousarray(np.concatenate(candidates) if count else np.zeros(0, CANDIDATE),
                                        dtype=CANDIDATE)
        else:
            counts = np.ascontiguousarray(counts, dtype=np.uint32)
            flat = np.ascontiguousarray(candidates, dtype=CANDIDATE)
        st = lib().brp_toplist_fold(self._t, arr, ptr(orb), ptr(flat), ptr(counts), count)
        if st:
            raise BrpError(st, "invalid compact candidate")
        return self

    def final(self):
        out = np.zeros(100, BANK_CANDIDATE)
        n = lib().brp_toplist_final(self._t, ptr(out))
        return out[:n].copy()
