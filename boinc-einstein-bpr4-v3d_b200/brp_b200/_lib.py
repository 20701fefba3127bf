"""ctypes binding of libbrp_cuda.so (the C ABI declared in include/brp_cuda.h).

The library is built in-tree by ``csrc/build.sh`` (``__graft_entry__.build()``
runs it); if it is missing it is built on first use.  There is no fallback:
without the library, or without a CUDA device, the calls raise.
"""
import ctypes
import os
import subprocess
import threading

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libbrp_cuda.so")
_lock = threading.Lock()
_lib = None


class BrpError(RuntimeError):
    """A non-zero status of the C ABI (status code in .status)."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class Params(ctypes.Structure):
    """brp_params: byte-identical to brp::Params (include/brp/science.hpp:8-17)."""
    _fields_ = [("n", ctypes.c_uint32), ("unpadded", ctypes.c_uint32), ("steps", ctypes.c_uint32),
                ("logn", ctypes.c_uint32), ("tau", ctypes.c_float), ("omega", ctypes.c_float),
                ("psi", ctypes.c_float), ("dt", ctypes.c_float), ("step_inv", ctypes.c_float),
                ("s0", ctypes.c_float), ("fundamental", ctypes.c_uint32), ("harmonic", ctypes.c_uint32),
                ("window", ctypes.c_uint32), ("stage", ctypes.c_uint32), ("threshold", ctypes.c_float * 5),
                ("capacity", ctypes.c_uint32), ("fft_n", ctypes.c_uint32), ("fft_base", ctypes.c_uint32),
                ("fft_radix", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("twiddle3", ctypes.c_uint32),
                ("twiddle_real", ctypes.c_uint32), ("result_slot", ctypes.c_uint32)]

    def copy(self):
        return Params.from_buffer_copy(self)

    def __repr__(self):
        return ("Params(n=%d, unpadded=%d, steps=%d, tau=%r, omega=%r, psi=%r, dt=%r, s0=%r, fundamental=%d, "
                "harmonic=%d, window=%d, threshold=%s, flags=%d)" % (
                    self.n, self.unpadded, self.steps, self.tau, self.omega, self.psi, self.dt, self.s0,
                    self.fundamental, self.harmonic, self.window, list(self.threshold), self.flags))


assert ctypes.sizeof(Params) == 108


def as_params(p):
    """Any 108-byte brp::Params-layout structure as a Params (copied)."""
    return Params.from_buffer_copy(bytes(p))


class Options(ctypes.Structure):
    _fields_ = [("workgroup", ctypes.c_uint32), ("tile", ctypes.c_uint32), ("batch", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("device", ctypes.c_int32), ("reserved", ctypes.c_uint32 * 3)]


class Timings(ctypes.Structure):
    _fields_ = [("wall_ms", ctypes.c_double), ("cpu_ms", ctypes.c_double), ("submit_ms", ctypes.c_double),
                ("stage_ms", ctypes.c_double * 4)]


CANDIDATE = np.dtype([("bin", "<u4"), ("level", "<u4"), ("power", "<f4"), ("reserved", "<u4")])
BANK_CANDIDATE = np.dtype([("power", "<f8"), ("period", "<f8"), ("tau", "<f8"), ("psi", "<f8"),
                           ("significance", "<f8"), ("harmonics", "<u4"), ("bin", "<u4")])

OPT = dict(software=1, stockham=2, radix4=4, packed=8, scatter=16, radix8=32, fused_power=64, radix8_store=128,
           plain=1 << 16)
STATUS_OVERFLOW, STATUS_RESAMPLE_OOB, STATUS_WAIT_TIMEOUT = 1, 2, 4
FLAG_FMA, FLAG_INDEX_FP64 = 2, 256

# Every symbol declared in include/brp_cuda.h.
EXPORTS = (
    "brp_cuda_create", "brp_cuda_destroy", "brp_cuda_set_templates", "brp_cuda_run", "brp_cuda_snapshot",
    "brp_cuda_candidates", "brp_cuda_device_info", "brp_cuda_allocated_bytes", "brp_cuda_profile_counters",
    "brp_cuda_last_error", "brp_cuda_bank_create", "brp_cuda_bank_destroy", "brp_cuda_bank_set_series",
    "brp_cuda_bank_run", "brp_cuda_bank_launch", "brp_cuda_bank_configure", "brp_cuda_bank_set_toplist_filter",
    "brp_cuda_fast_configs", "brp_cuda_bank_profile", "brp_cuda_bank_stream", "brp_cuda_bank_kernels_per_run",
    "brp_cuda_bank_last_error", "brp_host_parameters", "brp_host_resampling_steps", "brp_host_search_parameters",
    "brp_toplist_create", "brp_toplist_destroy", "brp_toplist_thresholds", "brp_toplist_retain",
    "brp_toplist_final", "brp_toplist_fold", "brp_cuda_search_static", "brp_cuda_search_static_error",
    "brp_cuda_preprocess", "brp_cuda_preprocess_dd", "brp_cuda_preprocess_error", "brp_host_read_zap",
    "brp_host_zap_noise", "brp_host_error", "brp_cuda_set_wait_limits", "brp_cuda_bank_set_wait_limits",
    "brp_cuda_debug_fail_allocation", "brp_cuda_bank_autotune", "brp_cuda_load_plan_cache",
    "brp_cuda_autotune_error", "brp_cuda_bank_submit", "brp_cuda_bank_wait",
)


def build(force=False):
    """Compile libbrp_cuda.so for sm_100a in-tree (nvcc cross-compiles without a GPU)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["sh", os.path.join(PKG_ROOT, "csrc", "build.sh"), LIB_PATH], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(LIB_PATH)
            P, vp, u32, u64 = ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
            L.brp_cuda_create.argtypes = [P, vp, u32, ctypes.POINTER(Options), ctypes.POINTER(vp)]
            L.brp_cuda_destroy.argtypes = [vp]
            L.brp_cuda_destroy.restype = None
            L.brp_cuda_set_templates.argtypes = [vp, P, u32]
            L.brp_cuda_run.argtypes = [vp, ctypes.POINTER(Timings), vp]
            L.brp_cuda_snapshot.argtypes = [vp, vp, vp, vp, vp]
            L.brp_cuda_candidates.argtypes = [vp, u32, vp, u32, ctypes.POINTER(u32)]
            L.brp_cuda_device_info.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
            L.brp_cuda_allocated_bytes.argtypes = [vp]
            L.brp_cuda_allocated_bytes.restype = u64
            L.brp_cuda_profile_counters.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t]
            L.brp_cuda_last_error.argtypes = [vp]
            L.brp_cuda_last_error.restype = ctypes.c_char_p
            L.brp_cuda_bank_create.argtypes = [u32, vp, vp, u32, u32, ctypes.c_int32, ctypes.POINTER(vp)]
            L.brp_cuda_bank_destroy.argtypes = [vp]
            L.brp_cuda_bank_destroy.restype = None
            L.brp_cuda_bank_set_series.argtypes = [vp, u32, vp]
            L.brp_cuda_bank_run.argtypes = [vp, vp, vp, u32, vp, u64, vp, vp]
            L.brp_cuda_bank_submit.argtypes = [vp, vp, vp, u32]
            L.brp_cuda_bank_wait.argtypes = [vp, vp, u64, vp, vp]
            L.brp_cuda_search_static.argtypes = [P, vp, vp, vp, u32, vp, vp, vp]
            L.brp_cuda_search_static_error.restype = ctypes.c_char_p
            L.brp_cuda_bank_launch.argtypes = [vp]
            L.brp_cuda_bank_configure.argtypes = [vp, u32, ctypes.c_int32, ctypes.c_int32, u32, u32]
            L.brp_cuda_bank_set_toplist_filter.argtypes = [vp, u32]
            L.brp_cuda_fast_configs.argtypes = [vp, vp, vp, u32]
            L.brp_cuda_bank_profile.argtypes = [vp, vp, vp]
            L.brp_cuda_bank_stream.argtypes = [vp]
            L.brp_cuda_bank_stream.restype = vp
            L.brp_cuda_bank_kernels_per_run.argtypes = [vp]
            L.brp_cuda_bank_kernels_per_run.restype = u32
            L.brp_cuda_bank_last_error.argtypes = [vp]
            L.brp_cuda_bank_last_error.restype = ctypes.c_char_p
            L.brp_host_parameters.argtypes = [u32, u32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                              ctypes.c_float, P]
            L.brp_host_resampling_steps.argtypes = [P]
            L.brp_host_search_parameters.argtypes = [u32, u32] + [ctypes.c_double] * 6 + [u32, P]
            L.brp_toplist_create.restype = vp
            L.brp_toplist_destroy.argtypes = [vp]
            L.brp_toplist_destroy.restype = None
            L.brp_toplist_thresholds.argtypes = [vp, P]
            L.brp_toplist_thresholds.restype = None
            L.brp_toplist_retain.argtypes = [vp, vp, u32, ctypes.c_double, ctypes.c_double, ctypes.c_double, P]
            L.brp_toplist_fold.argtypes = [vp, vp, vp, vp, vp, u32]
            L.brp_toplist_final.argtypes = [vp, vp]
            L.brp_toplist_final.restype = u32
            L.brp_cuda_set_wait_limits.argtypes = [vp, u32, ctypes.c_double]
            L.brp_cuda_bank_set_wait_limits.argtypes = [vp, u32, ctypes.c_double]
            L.brp_cuda_debug_fail_allocation.argtypes = [u32]
            L.brp_cuda_debug_fail_allocation.restype = None
            L.brp_cuda_bank_autotune.argtypes = [vp, vp, vp, u32, u32, vp, u32, ctypes.c_char_p, u32, vp, u32,
                                                 ctypes.POINTER(u32)]
            L.brp_cuda_load_plan_cache.argtypes = [ctypes.c_char_p]
            L.brp_cuda_autotune_error.restype = ctypes.c_char_p
            _lib = L
    return _lib


def check(status, message_fn):
    if status:
        raise BrpError(status, message_fn())


def fast_configs():
    """Compiled pass configurations: list of (id, L, kind) with kind 1 = pass 1,
    2 = pass 2, 3 = pass 1 with its first radix-16 stage on the tensor cores
    (chosen only by id)."""
    L = lib()
    n = L.brp_cuda_fast_configs(None, None, None, 0)
    ids = np.zeros(n, np.int32)
    lens = np.zeros(n, np.uint32)
    kinds = np.zeros(n, np.uint32)
    L.brp_cuda_fast_configs(ptr(ids), ptr(lens), ptr(kinds), n)
    return [(int(i), int(l), int(k)) for i, l, k in zip(ids, lens, kinds)]


def ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None
