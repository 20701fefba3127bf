"""brp_b200.GPU -- the reference's brp::GPU interface (include/brp/vulkan.hpp:12-29)
on the CUDA backend, through the C ABI.

Same constructor arguments, method names, argument meaning and error
behaviour: failures raise BrpError (the reference throws std::runtime_error).
"""
import ctypes
from collections import namedtuple

import numpy as np

from ._lib import CANDIDATE, OPT, BrpError, Options, Params, Timings, as_params, check, lib, ptr

Snapshot = namedtuple("Snapshot", "resampled power summed fft candidates")
RunTimings = namedtuple("RunTimings", "wall_ms cpu_ms submit_ms stage_ms template_stage_ms")
UINT32_MAX = 0xFFFFFFFF


class GPU:
    def __init__(self, params, input, workgroup=192, tile=512, batch=4, software=False, stockham=False,
                 radix4=False, packed=False, scatter=False, radix8=False, fused_power=False, radix8_store=False,
                 plain=False, device=-1, pass1=0, pass2=0):
        L = lib()
        self._ctx = None
        x = np.ascontiguousarray(input, dtype=np.float32)
        flags = 0
        for name, on in (("software", software), ("stockham", stockham), ("radix4", radix4), ("packed", packed),
                         ("scatter", scatter), ("radix8", radix8), ("fused_power", fused_power),
                         ("radix8_store", radix8_store), ("plain", plain)):
            if on:
                flags |= OPT[name]
        o = Options(workgroup, tile, batch, flags, device)
        o.reserved[0] = pass1 & 0xFFFFFFFF  # compiled pass configuration ids (-1: generic kernels)
        o.reserved[1] = pass2 & 0xFFFFFFFF
        ctx = ctypes.c_void_p()
        params = as_params(params)
        st = L.brp_cuda_create(ctypes.byref(params), ptr(x), x.size, ctypes.byref(o), ctypes.byref(ctx))
        check(st, lambda: L.brp_cuda_last_error(None).decode())
        self._ctx = ctx
        self.params = params.copy()
        self.batch = batch
        self._templates = [params.copy()]

    def _err(self):
        return lib().brp_cuda_last_error(self._ctx).decode()

    def close(self):
        if self._ctx:
            lib().brp_cuda_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_template(self, p):
        self.set_templates([p])

    def set_templates(self, templates):
        arr = (Params * len(templates))(*[as_params(t) for t in templates])
        check(lib().brp_cuda_set_templates(self._ctx, arr, len(templates)), self._err)
        self._templates = [t.copy() for t in templates]

    def run(self):
        t = Timings()
        per = np.zeros(4 * len(self._templates), np.float64)
        check(lib().brp_cuda_run(self._ctx, ctypes.byref(t), ptr(per)), self._err)
        return RunTimings(t.wall_ms, t.cpu_ms, t.submit_ms, list(t.stage_ms), per.reshape(-1, 4))

    def snapshot(self):
        p = self._templates[-1]
        r = np.empty(p.n, np.float32)
        f = np.empty(2 * (p.n // 2 + 1), np.float32)
        w = np.empty(p.n // 2, np.float32)
        s = np.empty(5 * p.fundamental, np.float32)
        check(lib().brp_cuda_snapshot(self._ctx, ptr(r), ptr(f), ptr(w), ptr(s)), self._err)
        return Snapshot(r, w, s, f.view(np.complex64), self.candidates())

    def candidates(self, slot=UINT32_MAX):
        n = ctypes.c_uint32()
        check(lib().brp_cuda_candidates(self._ctx, slot, None, 0, ctypes.byref(n)), self._err)
        out = np.empty(n.value, CANDIDATE)
        check(lib().brp_cuda_candidates(self._ctx, slot, ptr(out), n.value, ctypes.byref(n)), self._err)
        return out

    def set_wait_limits(self, device_polls=1 << 22, host_seconds=300.0):
        """Bounds of run()'s waits (the reference waits without a bound,
        src/vulkan.cpp:306): the host deadline, and the poll bound of a kernel's
        first wait for its own asynchronous work (0 gives up at once)."""
        check(lib().brp_cuda_set_wait_limits(self._ctx, device_polls, host_seconds), self._err)

    def device_info(self):
        buf = ctypes.create_string_buffer(1024)
        check(lib().brp_cuda_device_info(self._ctx, buf, len(buf)), self._err)
        return buf.value.decode()

    def allocated_bytes(self):
        return int(lib().brp_cuda_allocated_bytes(self._ctx))

    def profile_counters(self):
        buf = ctypes.create_string_buffer(4096)
        check(lib().brp_cuda_profile_counters(self._ctx, buf, len(buf)), self._err)
        return buf.value.decode()
